/*
 * bp_oracle.c -- CPU restatement of mmNorm's SAR backprojection and surface-normal
 * vote, in FP64.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the
 * CPU-baseline leg of the benchmark call this code as the checker.  The product
 * path (mmnorm_b200) never links or calls it.
 *
 * Every function works on an explicit list of voxel centres, so the same code
 * serves a full grid (tiny cases) and a seeded random subset of a large grid.
 *
 * Reference arithmetic followed (paths relative to the mmNorm repository):
 *   - round-trip distance TX->voxel->RX, RX offset, TI 0.15 m:
 *       src/data_processing/cuda/imaging_gpu.cu:65-88
 *   - full matched filter, phase -2*pi*d*(1/lambda + j*slope/c):
 *       src/data_processing/cuda/imaging_gpu.cu:106-117
 *   - interpolated mode (range check, bin = floor(d/fft_spacing/2), one phasor):
 *       src/data_processing/cuda/imaging_gpu.cu:90-105
 *   - normal vote sum_i Re(c_i conj(I))/|I| * (tx_i + o/2 - v):
 *       src/data_processing/cuda/surface_normal_est.cu:84-145
 *
 * All arithmetic is double precision on float32 inputs promoted to double; sine
 * and cosine come from libm.  phase_mode 1 replaces the per-sample libm call by
 * an FP64 rotation re-anchored with libm every 32 samples (error ~1e-14), which is
 * an order of magnitude faster for the large accuracy reports.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#define ORC_C 2.99792458e8
#define ORC_PI 3.14159265358979323846264338327950288

static inline double orc_dist(double vx, double vy, double vz, const float *a,
                              const float *o, int is_ti) {
    double dx = vx - (double)a[0], dy = vy - (double)a[1], dz = vz - (double)a[2];
    double fwd = sqrt(dx * dx + dy * dy + dz * dz);
    double bx = dx - (double)o[0], by = dy - (double)o[1], bz = dz - (double)o[2];
    double back = sqrt(bx * bx + by * by + bz * bz);
    double d = fwd + back;
    if (is_ti) d += 0.15;
    return d;
}

/*
 * Full matched-filter image and vote.
 *   img[v]   = sum_i sum_j m[i,j] * exp(-i*2*pi*d_i(v)*(1/lambda + j*slope/c))
 *   vote[v]  = sum_i c_i(v) * (tx_i + o_{i%R}/2 - v)          (complex 3-vector)
 * meas is complex64 interleaved, [na, ns]; img is complex128 interleaved [nv];
 * vote (may be NULL) is [nv, 3] complex128 interleaved.
 */
void orc_full(int64_t nv, const float *vx, const float *vy, const float *vz,
              int64_t na, int32_t nrx, const float *ant, const float *rxo,
              int32_t ns, const float *meas, double wavelength, double slope,
              int32_t is_ti, int32_t phase_mode, double *img, double *vote) {
    const double k0 = 2.0 * ORC_PI / wavelength;
    const double kd = 2.0 * ORC_PI * slope / ORC_C;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t v = 0; v < nv; ++v) {
        double x = vx[v], y = vy[v], z = vz[v];
        double ir = 0, ii = 0;
        double w[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t i = 0; i < na; ++i) {
            const float *a = ant + 3 * i;
            const float *o = rxo + 3 * (i % nrx);
            double d = orc_dist(x, y, z, a, o, is_ti);
            const float *m = meas + 2 * i * (int64_t)ns;
            double cr = 0, ci = 0;
            if (phase_mode == 0) {
                for (int32_t j = 0; j < ns; ++j) {
                    double ph = -d * (k0 + (double)j * kd);
                    double c = cos(ph), s = sin(ph);
                    double mr = m[2 * j], mi = m[2 * j + 1];
                    cr += mr * c - mi * s;
                    ci += mr * s + mi * c;
                }
            } else {
                double zr = cos(-d * kd), zi = sin(-d * kd);
                double pr = 0, pi = 0;
                for (int32_t j = 0; j < ns; ++j) {
                    if ((j & 31) == 0) {
                        double ph = -d * (k0 + (double)j * kd);
                        pr = cos(ph);
                        pi = sin(ph);
                    }
                    double mr = m[2 * j], mi = m[2 * j + 1];
                    cr += mr * pr - mi * pi;
                    ci += mr * pi + mi * pr;
                    double t = pr * zr - pi * zi;
                    pi = pr * zi + pi * zr;
                    pr = t;
                }
            }
            ir += cr;
            ii += ci;
            if (vote) {
                double ux = (double)a[0] + (double)o[0] / 2 - x;
                double uy = (double)a[1] + (double)o[1] / 2 - y;
                double uz = (double)a[2] + (double)o[2] / 2 - z;
                w[0] += cr * ux; w[1] += ci * ux;
                w[2] += cr * uy; w[3] += ci * uy;
                w[4] += cr * uz; w[5] += ci * uz;
            }
        }
        img[2 * v] = ir;
        img[2 * v + 1] = ii;
        if (vote)
            for (int k = 0; k < 6; ++k) vote[6 * v + k] = w[k];
    }
}

/*
 * Interpolated-mode contribution c_i(v) (imaging_gpu.cu:90-105): the range-FFT bin
 * floor(d/fft_spacing/2) of antenna i times exp(-i*2*pi*d/lambda); skipped when
 * d < 0 or d > fft_spacing*nbins.  dist_mode 0 computes d in FP64; dist_mode 1
 * computes it in float32 (no contraction) as the reference's float code does, so
 * the bin choice follows the reference's rounding up to FMA contraction.
 * Returns 0 when the antenna is skipped.
 */
static inline int orc_interp_contrib(double x, double y, double z, const float *a,
                                     const float *o, int is_ti, int dist_mode,
                                     const float *m, int32_t nb, double wavelength,
                                     double fft_spacing, double *cr, double *ci) {
    double d;
    if (dist_mode == 0) {
        d = orc_dist(x, y, z, a, o, is_ti);
    } else {
        volatile float dx = (float)x - a[0], dy = (float)y - a[1], dz = (float)z - a[2];
        volatile float fsq = dx * dx;
        fsq = fsq + dy * dy;
        fsq = fsq + dz * dz;
        float fwd = sqrtf(fsq);
        volatile float bx = dx - o[0], by = dy - o[1], bz = dz - o[2];
        volatile float bsq = bx * bx;
        bsq = bsq + by * by;
        bsq = bsq + bz * bz;
        float back = sqrtf(bsq);
        float df = fwd + back;
        if (is_ti) df += 0.15f;
        d = df;
    }
    float fsp = (float)fft_spacing;
    if (d < 0 || d > (double)(fsp * (float)nb)) return 0;
    int bin;
    if (dist_mode == 0)
        bin = (int)floor(d / fft_spacing / 2);
    else
        bin = (int)floorf((float)d / fsp / 2);
    if (bin < 0 || bin >= nb) return 0; /* unreachable for valid inputs */
    double ph = -2.0 * ORC_PI * d / wavelength;
    double c = cos(ph), s = sin(ph);
    double mr = m[2 * bin], mi = m[2 * bin + 1];
    *cr = mr * c - mi * s;
    *ci = mr * s + mi * c;
    return 1;
}

/* Interpolated-mode image (and, if vote != NULL, the fused vote vector). */
void orc_interp(int64_t nv, const float *vx, const float *vy, const float *vz,
                int64_t na, int32_t nrx, const float *ant, const float *rxo,
                int32_t nb, const float *meas, double wavelength, double fft_spacing,
                int32_t is_ti, int32_t dist_mode, double *img, double *vote) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t v = 0; v < nv; ++v) {
        double x = vx[v], y = vy[v], z = vz[v];
        double ir = 0, ii = 0, w[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t i = 0; i < na; ++i) {
            const float *a = ant + 3 * i;
            const float *o = rxo + 3 * (i % nrx);
            double cr, ci;
            if (!orc_interp_contrib(x, y, z, a, o, is_ti, dist_mode,
                                    meas + 2 * i * (int64_t)nb, nb, wavelength,
                                    fft_spacing, &cr, &ci))
                continue;
            ir += cr;
            ii += ci;
            if (vote) {
                double ux = (double)a[0] + (double)o[0] / 2 - x;
                double uy = (double)a[1] + (double)o[1] / 2 - y;
                double uz = (double)a[2] + (double)o[2] / 2 - z;
                w[0] += cr * ux; w[1] += ci * ux;
                w[2] += cr * uy; w[3] += ci * uy;
                w[4] += cr * uz; w[5] += ci * uz;
            }
        }
        img[2 * v] = ir;
        img[2 * v + 1] = ii;
        if (vote)
            for (int k = 0; k < 6; ++k) vote[6 * v + k] = w[k];
    }
}

/*
 * Normal vote for a list of valid voxels with a given image value per voxel
 * (surface_normal_est.cu:84-145):  n = sum_i Re(c_i conj(I))/|I| * (tx_i + o/2 - v),
 * c_i the interpolated-mode contribution.  normals is [nv, 3] double.
 */
void orc_sn_interp(int64_t nv, const float *vx, const float *vy, const float *vz,
                   const float *img_r, const float *img_i, int64_t na, int32_t nrx,
                   const float *ant, const float *rxo, int32_t nb, const float *meas,
                   double wavelength, double fft_spacing, int32_t is_ti,
                   int32_t dist_mode, double *normals) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t v = 0; v < nv; ++v) {
        double x = vx[v], y = vy[v], z = vz[v];
        double ir = img_r[v], ii = img_i[v];
        double mag = sqrt(ir * ir + ii * ii);
        double n0 = 0, n1 = 0, n2 = 0;
        for (int64_t i = 0; i < na; ++i) {
            const float *a = ant + 3 * i;
            const float *o = rxo + 3 * (i % nrx);
            double cr, ci;
            if (!orc_interp_contrib(x, y, z, a, o, is_ti, dist_mode,
                                    meas + 2 * i * (int64_t)nb, nb, wavelength,
                                    fft_spacing, &cr, &ci))
                continue;
            double wgt = (cr * ir + ci * ii) / mag;
            n0 += ((double)a[0] + (double)o[0] / 2 - x) * wgt;
            n1 += ((double)a[1] + (double)o[1] / 2 - y) * wgt;
            n2 += ((double)a[2] + (double)o[2] / 2 - z) * wgt;
        }
        normals[3 * v] = n0;
        normals[3 * v + 1] = n1;
        normals[3 * v + 2] = n2;
    }
}

/*
 * Adjoint (backward) of orc_full for the loss-gradient check.  Given upstream
 * gradients gI[v] (complex) and gW[v,k] (complex, k=x,y,z) in the torch
 * convention (grad = dL/dRe + i dL/dIm), returns
 *   gmeas[i,j] = sum_v G_i(v) * exp(+i*phi_ij(v)),  G_i(v) = gI + sum_k gW_k u_ik
 *   gpos[i,k]  = d L / d (tx_i)_k, for a per-antenna offset added to the TX (and
 *                with it the RX) position.
 * Slow reference for small cases only.
 */
void orc_full_backward(int64_t nv, const float *vx, const float *vy, const float *vz,
                       int64_t na, int32_t nrx, const float *ant, const float *rxo,
                       int32_t ns, const float *meas, double wavelength, double slope,
                       int32_t is_ti, const double *gI, const double *gW,
                       double *gmeas, double *gpos) {
    const double k0 = 2.0 * ORC_PI / wavelength;
    const double kd = 2.0 * ORC_PI * slope / ORC_C;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < na; ++i) {
        const float *a = ant + 3 * i;
        const float *o = rxo + 3 * (i % nrx);
        const float *m = meas + 2 * i * (int64_t)ns;
        double *gm = gmeas + 2 * i * (int64_t)ns;
        for (int32_t j = 0; j < 2 * ns; ++j) gm[j] = 0;
        double gp[3] = {0, 0, 0};
        for (int64_t v = 0; v < nv; ++v) {
            double x = vx[v], y = vy[v], z = vz[v];
            double dx = x - (double)a[0], dy = y - (double)a[1], dz = z - (double)a[2];
            double fwd = sqrt(dx * dx + dy * dy + dz * dz);
            double bx = dx - (double)o[0], by = dy - (double)o[1], bz = dz - (double)o[2];
            double back = sqrt(bx * bx + by * by + bz * bz);
            double d = fwd + back + (is_ti ? 0.15 : 0.0);
            double u[3] = {(double)a[0] + (double)o[0] / 2 - x,
                           (double)a[1] + (double)o[1] / 2 - y,
                           (double)a[2] + (double)o[2] / 2 - z};
            double Gr = gI[2 * v], Gi = gI[2 * v + 1];
            for (int k = 0; k < 3; ++k) {
                Gr += gW[6 * v + 2 * k] * u[k];
                Gi += gW[6 * v + 2 * k + 1] * u[k];
            }
            double cr = 0, ci = 0, dcr = 0, dci = 0; /* c and dc/dd */
            for (int32_t j = 0; j < ns; ++j) {
                double kj = k0 + (double)j * kd;
                double ph = -d * kj;
                double c = cos(ph), s = sin(ph);
                double mr = m[2 * j], mi = m[2 * j + 1];
                double tr = mr * c - mi * s, ti = mr * s + mi * c;
                cr += tr; ci += ti;
                /* d/dd of m*exp(-i d kj) = -i kj * term */
                dcr += kj * ti;
                dci += -kj * tr;
                /* gmeas += G * conj(exp(i ph)) */
                gm[2 * j] += Gr * c + Gi * s;
                gm[2 * j + 1] += Gi * c - Gr * s;
            }
            /* dL/dd = Re(conj(G) * dc/dd) */
            double dLdd = Gr * dcr + Gi * dci;
            /* dd/dtx = -(v-tx)/|v-tx| - (v-tx-o)/|v-tx-o| */
            double dd[3] = {-dx / fwd - bx / back, -dy / fwd - by / back,
                            -dz / fwd - bz / back};
            for (int k = 0; k < 3; ++k) {
                /* u_k depends on tx_k with derivative 1: dL/du_k = Re(conj(gW_k) c) */
                double dLdu = gW[6 * v + 2 * k] * cr + gW[6 * v + 2 * k + 1] * ci;
                gp[k] += dLdd * dd[k] + dLdu;
            }
        }
        for (int k = 0; k < 3; ++k) gpos[3 * i + k] = gp[k];
    }
}

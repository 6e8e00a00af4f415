// bp_kernels.cuh -- kernel parameter blocks and launch helpers shared by the
// kernel files and the C ABI (capi.cu).
#pragma once
#include <atomic>

#include "mmn_internal.cuh"

namespace mmn {

// ------------------------------------------------------------- full-mode forward
struct FwdParams {
    const float *x_locs, *y_locs, *z_locs;
    int32_t nx, ny, nz;
    int64_t nvox;          // voxels in the whole grid
    int64_t vox_start;     // first voxel of this launch
    int64_t vox_count;     // voxels in this launch (tiles cover [vox_start, +vox_count))
    const AntRec *ant;     // [num_ant]
    const void *meas;      // [num_ant, fp] samples in the kernel form's layout (8 or 16 B each)
    int32_t num_ant;
    int32_t fp;
    int32_t ant_per_stage; // antennas per shared-memory stage
    int32_t nsmp;          // samples per row before padding (F); 0: fp (the second-order
                           // forms skip the padded zeros of a row's last block)
    const int32_t *mono_flag; // device word: 1 when all RX offsets are zero
    double k0, kd;         // 2*pi/lambda, 2*pi*slope/c
    double t0, tblk;       // 1/lambda and 32*slope/c: turns per metre of range
    double tsmp;           // slope/c: turns per metre of range per sample
    double ti;             // 0.15 or 0
    int32_t num_tiles;
    int32_t num_splits;
    int32_t ant_per_split;
    int32_t pad0;
    float2 *image;         // [nvox] complex64 or null
    float2 *vote;          // [3, nvox] or null
    float *out_r, *out_i;  // [nvox] SoA image (reference layout) or null
    float4 *partial;       // [num_splits, vox_count, 2] (num_splits > 1)
    int32_t *status;
};

struct FwdVariant {
    int t;      // voxels per thread
    int nt;     // threads per CTA
    bool plain; // PLAIN form
    int esz;    // staged bytes per antenna-sample: 8 or 16
    const void *fn;
    const char *name;
    int layout; // staged sample layout (stage_meas): 0 (re,im), 1 (re,re,im,im), 2 antenna pairs
    const void *persistent_fn;  // bp_fwd_persistent instantiation of the same form, or null
    int max_stage_bytes;        // cap on one shared-memory stage; 0: the library default
};

// Batched (persistent) forward: per-object FwdParams and a cost-sorted work list.
struct BatchParams {
    const FwdParams *objs;  // [num_objects]
    const int4 *items;      // [num_items] (object, tile, split, -)
    int32_t num_items;
    int32_t pad0;
    int *counter;           // work-list cursor, zeroed before each launch
};

const FwdVariant *fwd_variants(int *count);
cudaError_t launch_fwd(const FwdVariant &var, const FwdParams &p, size_t smem,
                       cudaStream_t stream);
cudaError_t launch_reduce(const FwdParams &p, cudaStream_t stream);
cudaError_t launch_prep_antennas(const float *ant, const float *rxo, int R, const float *pos_off,
                                 int A, int A_pad, AntRec *out, int32_t *mono_flag,
                                 cudaStream_t stream);
cudaError_t launch_stage_meas(const float *src, const float *im, int A, int F, int Fp,
                              int layout, void *dst, cudaStream_t stream);

// ------------------------------------------------------------------- backward
struct BwdParams {
    FwdParams f;               // geometry, antenna records, staged (kappa*m, m) samples, tiles
    const float2 *grad_image;  // [nvox] complex64 dL/dI (torch convention)
    const float2 *grad_vote;   // [3, nvox] complex64 dL/dW, or null
    float *pos_partial;        // [num_tiles, a_pad, 3] per-tile position-gradient sums
    const float4 *vox_rec;     // [nvox, 3] voxel records (x, y, z, -), (gI, gWx), (gWy, gWz)
    float2 *grad_meas;         // [num_ant_real, num_samples] complex64
    float *grad_pos;           // [num_ant_real, 3]
    int32_t num_samples;       // unpadded F
    int32_t num_ant_real;      // A before padding
    int32_t num_items;         // num_ant_real * (fp / 32): (antenna, 32-sample block) pairs
    int32_t meas_splits;       // voxel ranges of the measurement pass (1: no partial sums)
    float2 *meas_partial;      // [meas_splits, num_ant_real, num_samples] if meas_splits > 1
    int64_t vox_per_split;     // voxels per measurement-pass range (a multiple of 512)
    int32_t nu_n;              // interpolation-form position pass: grid cells N = 2F
    int32_t pad_nu;
    double nu_u;               // slope / c: turns per sample per metre of range
    double nu_k0c;             // 2pi (1/lambda + J0 slope/c), J0 = F/2: anchor phase per metre
};

// Interpolation-form position pass (bp_nufft.cu): kernel width in grid cells, and the
// length of one antenna's staged grid row (N + W - 1 cells, so that no tap run wraps).
constexpr int kNuW = 8;
__host__ __device__ constexpr int nufft_row(int n) { return n + kNuW - 1; }
// Row length of the forward's (G.re, G.im) rows: nufft_row rounded up to an even number of
// 8-byte cells, so that every row, stage and bulk copy stays a multiple of 16 bytes.
__host__ __device__ constexpr int nufft_row_fwd(int n) { return (nufft_row(n) + 1) & ~1; }

cudaError_t launch_bwd_stage(const float *meas, int A, int F, int Fp, double k0, double kd,
                             int layout, void *dst, cudaStream_t stream);
cudaError_t launch_bwd_vox_rec(const BwdParams &bp, float4 *dst, cudaStream_t stream);
cudaError_t launch_bwd_pos(const BwdParams &bp, int variant, size_t smem, cudaStream_t stream);
cudaError_t launch_bwd_pos_reduce(const BwdParams &bp, cudaStream_t stream);
cudaError_t launch_bwd_meas(const BwdParams &bp, cudaStream_t stream);
// voxel ranges for the measurement pass: fills the GPU in whole waves of CTAs
int bwd_meas_splits(int num_ant, int fp, int64_t nvox);
const void *bwd_pos_kernel_ptr(int variant, int *threads, int *voxels_per_thread);
// position pass for losses without a vote term (launch_bwd_pos with variant -1)
const void *bwd_pos_img_kernel_ptr(int *threads, int *voxels_per_thread);
// interpolation-form position pass (vote: the loss has a vote term) and its per-antenna
// grids: tables (tw [N] double2, 16-byte aligned; sc [F] doubles) and rows
// [A][nufft_row(N)] float4
const void *bwd_pos_nufft_kernel_ptr(int variant, bool vote, int *threads, int *voxels_per_thread,
                                     int *stage_cap_bytes);
int bwd_pos_nufft_num_variants();
// Interpolation-form measurement pass.
struct NuMeasParams {
    const AntRec *ant;
    const float4 *vox;        // [nvox][5] records (nufft_vox_kernel)
    const int32_t *mono_flag;
    float2 *part;             // [ranges][num_ant][mrow] per-range antenna grids
    const double *sc;         // [F] 1/phihat((j - J0)/N)
    const double2 *tw;        // [N] e^{-2pi i k/N}
    float2 *grad_meas;        // [num_ant][F]
    int64_t nvox, vox_per_range;
    double ti, uq, k0c;       // 0.15 or 0; slope/c; 2pi(1/lambda + J0 slope/c)
    int32_t num_ant, n, mrow, ranges, F, J0;  // mrow = N + 16 cells
};
// forward in interpolation form (bp_fwd_nufft_kernel; BwdParams carries the nu fields)
const void *fwd_nufft_kernel_ptr(int *threads, int *voxels_per_thread);
size_t nufft_meas_smem(int mrow);
int nufft_meas_warps();
const void *nufft_meas_kernel_ptr();
cudaError_t launch_nufft_meas(const NuMeasParams &q, const FwdParams &p,
                              const float2 *grad_image, const float2 *grad_vote, float4 *rec,
                              cudaStream_t stream);
const char *bwd_pos_nufft_variant_name(int variant);  // null for a bad index
cudaError_t launch_nufft_tables(int F, int N, int J0, double *sc, double2 *tw,
                                cudaStream_t stream);
cudaError_t launch_nufft_grid(const float *meas, int A, int F, int N, int J0, double k0,
                              double kd, const double *sc, const double2 *tw, void *rows,
                              bool fwd_only, cudaStream_t stream);

// ---------------------------------------------------------- interpolated mode
struct InterpParams {
    const float *x_locs, *y_locs, *z_locs;
    int32_t nx, ny, nz;
    int32_t num_ant, num_rx, nbins;
    const float *ant;        // [num_ant, 3]
    const float *rxo;        // [num_rx, 3]
    const float2 *meas;      // complex64 [num_ant, nbins] (or null when SoA is used)
    const float *meas_r;     // SoA planes (reference layout) or null
    const float *meas_i;
    float fft_spacing, wavelength;
    int32_t is_ti;
    int32_t pad0;
    // image pass: voxels [start, start + count)
    int64_t start, count;
    float *out_r, *out_i;    // SoA outputs (reference layout) or null
    float2 *image;           // complex64 output or null
    float2 *vote;            // fused vote [3, V] (image pass) or null
    int64_t nvox;
    // normal pass (cuda_sn_est): valid voxel lists
    const int *vidx_x, *vidx_y, *vidx_z;
    const float *img_r, *img_i;
    float *n_x, *n_y, *n_z;
    int32_t num_valid;
    int32_t pad1;
    // fast form only: 1/lambda split into two floats (hi + lo) and 1/(2 fft_spacing)
    float inv_lambda_hi, inv_lambda_lo, half_inv_fsp;
    int32_t mono;            // 1 when every RX offset is zero (fast form)
};

cudaError_t launch_interp_image(const InterpParams &p, cudaStream_t stream);
cudaError_t launch_interp_normals(const InterpParams &p, cudaStream_t stream);
// fast form of both passes: same path length and range bin as the reference, the
// phasor from a wrapped FP32 turn count and the hardware sine/cosine
cudaError_t launch_interp_image_fast(const InterpParams &p, cudaStream_t stream);
extern std::atomic<int> g_interp_fast_form;  // form of the fast image pass (bp_interp.cu)
cudaError_t launch_interp_normals_fast(const InterpParams &p, cudaStream_t stream);

// --------------------------------------------------------------------- epilogue
cudaError_t launch_max_abs(int64_t nvox, const float2 *image, unsigned int *max_bits,
                           cudaStream_t stream);
cudaError_t launch_normals_from_max(int64_t nvox, const float2 *image, const float2 *vote,
                                    float filter_percent, float *normals, uint8_t *mask,
                                    float *raw, const unsigned int *max_bits,
                                    cudaStream_t stream);
cudaError_t launch_normals(int64_t nvox, const float2 *image, const float2 *vote,
                           float filter_percent, float *normals, uint8_t *mask, float *raw,
                           unsigned int *max_bits, cudaStream_t stream);

}  // namespace mmn

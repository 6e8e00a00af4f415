// capi.cu -- extern "C" entry points declared in include/mmnorm_b200.h.
//
// Host-side planning for the fused forward pass:
//   * measurement rows are padded to Fp = roundup(F, 32) samples (zero samples add
//     nothing) and must sit 16-byte aligned for the bulk copies, else they are copied
//     into the workspace;
//   * antennas per shared-memory stage = 48 KB / (64 + 8*Fp), at most 16;
//   * voxel tiles of NT*T voxels; when there are too few tiles to fill the GPU, the
//     antenna range is split S ways (S chosen by a wave-quantisation cost model over
//     the occupancy-derived CTA slots) and the S partial sums are reduced in split order.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <vector>

#include <cuda.h>  // driver types for the context-id lookup (entry points come from the runtime)

#include "bp_kernels.cuh"

using namespace mmn;

namespace {

constexpr size_t kAlign = 256;
constexpr int kMaxStageBytes = 48 * 1024;
constexpr int kMaxFp = 24576;  // one antenna row per stage still fits in shared memory
constexpr int kMaxFastBins = 1 << 22;  // fast interpolated form: rounding-constant bins

inline size_t align_up(size_t x, size_t a = kAlign) { return (x + a - 1) / a * a; }

std::atomic<int> g_variant[2] = {{-1}, {-1}};  // selected variant per MIXED / PLAIN; -1: first

struct FwdPlan {
    const FwdVariant *var;
    int fp, ant_per_stage, tiles, splits, ant_per_split, a_pad;
    size_t smem;
    int64_t vox_start, vox_count;
    bool copy_meas;
    size_t off_ant, off_meas, off_partial, total;
};

int variant_index_for(int mode) { return g_variant[mode == MMN_MODE_PLAIN ? 1 : 0].load(); }

bool misaligned(const void *q, uintptr_t bytes) {
    return (reinterpret_cast<uintptr_t>(q) & (bytes - 1)) != 0;
}

// Any of the 4-byte (float, int) arrays of the reference-signature entry points off a
// 4-byte boundary.
bool any_misaligned4(std::initializer_list<const void *> ptrs) {
    for (const void *q : ptrs)
        if (misaligned(q, 4)) return true;
    return false;
}

int check_problem(const mmn_problem *p, int mode) {
    if (!p) return MMN_ERR_NULL_POINTER;
    if (mode != MMN_MODE_MIXED && mode != MMN_MODE_PLAIN && mode != MMN_MODE_INTERP &&
        mode != MMN_MODE_INTERP_FAST)
        return MMN_ERR_INVALID_ARGUMENT;
    if (p->num_x < 1 || p->num_y < 1 || p->num_z < 1) return MMN_ERR_INVALID_ARGUMENT;
    if (p->num_antennas < 0 || p->num_rx < 1 || p->num_samples < 1)
        return MMN_ERR_INVALID_ARGUMENT;
    if (!(p->wavelength > 0.0) || !std::isfinite(p->wavelength) || !std::isfinite(p->slope))
        return MMN_ERR_INVALID_ARGUMENT;
    if ((mode == MMN_MODE_INTERP || mode == MMN_MODE_INTERP_FAST) && !(p->fft_spacing > 0.0))
        return MMN_ERR_INVALID_ARGUMENT;
    if (mode == MMN_MODE_INTERP_FAST && p->num_samples > kMaxFastBins) return MMN_ERR_TOO_LARGE;
    if (!p->x_locs || !p->y_locs || !p->z_locs) return MMN_ERR_NULL_POINTER;
    if (p->num_antennas > 0 && (!p->antenna_locs || !p->rx_offsets || !p->meas))
        return MMN_ERR_NULL_POINTER;
    // element alignment: the kernels load float arrays as 4-byte words and a complex64
    // sample as one 8-byte word, so a pointer off that grid is refused here rather than
    // reaching a misaligned device load
    if (misaligned(p->x_locs, 4) || misaligned(p->y_locs, 4) || misaligned(p->z_locs, 4) ||
        misaligned(p->pos_offsets, 4))
        return MMN_ERR_INVALID_ARGUMENT;
    if (p->num_antennas > 0 && (misaligned(p->antenna_locs, 4) ||
                                misaligned(p->rx_offsets, 4) || misaligned(p->meas, 8)))
        return MMN_ERR_INVALID_ARGUMENT;
    return MMN_OK;
}

int plan_forward(int64_t nvox, int64_t vox_start, int64_t vox_count, int A, int F, int mode,
                 bool meas_aligned, bool want_partial_space, FwdPlan *pl) {
    int nvar = 0;
    const FwdVariant *vars = fwd_variants(&nvar);
    int vi = variant_index_for(mode);
    if (vi < 0 || vi >= nvar || vars[vi].plain != (mode == MMN_MODE_PLAIN)) {
        vi = 0;
        while (vi < nvar && vars[vi].plain != (mode == MMN_MODE_PLAIN)) ++vi;
    }
    pl->var = &vars[vi];
    const bool pairs = pl->var->layout == 2;
    pl->a_pad = pairs ? A + (A & 1) : A;
    A = pl->a_pad;
    pl->fp = (F + kBlockF - 1) / kBlockF * kBlockF;
    if (pl->fp > kMaxFp) return MMN_ERR_TOO_LARGE;
    const int esz = pl->var->esz;
    const int rec = (int)sizeof(AntRec) + pl->fp * esz;
    const int cap = pl->var->max_stage_bytes > 0 ? pl->var->max_stage_bytes : kMaxStageBytes;
    pl->ant_per_stage = std::max(1, std::min(16, cap / rec));
    if (pairs) pl->ant_per_stage = std::max(2, pl->ant_per_stage & ~1);
    pl->smem = 128 + 2 * (size_t)pl->ant_per_stage * rec + (pl->var->plain ? pl->fp * 4 : 0);
    pl->vox_start = vox_start;
    pl->vox_count = vox_count;
    const int64_t per_tile = (int64_t)pl->var->nt * pl->var->t;
    const int64_t tiles = (vox_count + per_tile - 1) / per_tile;
    if (tiles > (int64_t)1 << 30) return MMN_ERR_TOO_LARGE;
    pl->tiles = (int)std::max<int64_t>(1, tiles);

    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (pl->smem > 48 * 1024)
        cudaFuncSetAttribute(pl->var->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pl->smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pl->var->fn, pl->var->nt,
                                                      pl->smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int64_t slots = (int64_t)sms * per_sm;
    // split count: minimise waves * antennas-per-CTA, with a 2 % charge per extra split
    int best_s = 1;
    double best_cost = 1e300;
    const int max_s = std::max(1, std::min(64, (A + pl->ant_per_stage - 1) / pl->ant_per_stage));
    for (int s = 1; s <= max_s; ++s) {
        const int64_t ctas = (int64_t)pl->tiles * s;
        const double waves = (double)((ctas + slots - 1) / slots);
        const double cost = waves * std::ceil((double)A / s) * (1.0 + 0.02 * (s - 1));
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best_s = s;
        }
        if (ctas >= 8 * slots) break;
    }
    pl->splits = best_s;
    pl->ant_per_split = A > 0 ? (A + best_s - 1) / best_s : 0;
    // keep whole stages per split when possible (fewer partial stages)
    if (best_s > 1) {
        int aps = (pl->ant_per_split + pl->ant_per_stage - 1) / pl->ant_per_stage * pl->ant_per_stage;
        pl->ant_per_split = aps;
        pl->splits = (A + aps - 1) / aps;
    }
    pl->copy_meas = pl->var->layout != 0 || !meas_aligned || pl->fp != F;
    size_t off = kStatusBytes;
    pl->off_ant = off;
    off = align_up(off + (size_t)A * sizeof(AntRec));  // A is the padded count here
    pl->off_meas = off;
    if (pl->copy_meas) off = align_up(off + (size_t)A * pl->fp * esz);
    pl->off_partial = off;
    if (pl->splits > 1 || want_partial_space)
        off = align_up(off + (size_t)pl->splits * (size_t)vox_count * 8 * sizeof(float));
    pl->total = off;
    return MMN_OK;
}

int run_forward(const FwdPlan &pl, const mmn_problem *p, const float *meas_r,
                const float *meas_i, float2 *image, float2 *vote, float *out_r, float *out_i,
                unsigned char *ws, cudaStream_t stream) {
    const int A = p->num_antennas;
    const int F = p->num_samples;
    cudaError_t e = cudaMemsetAsync(ws, 0, 16, stream);
    if (e != cudaSuccess) return MMN_ERR_CUDA;
    AntRec *ant = reinterpret_cast<AntRec *>(ws + pl.off_ant);
    int32_t *hdr = reinterpret_cast<int32_t *>(ws);
    e = launch_prep_antennas(p->antenna_locs, p->rx_offsets, p->num_rx, p->pos_offsets, A,
                             pl.a_pad, ant, hdr + 1, stream);
    if (e != cudaSuccess) return MMN_ERR_CUDA;
    const void *meas = p->meas;
    if (meas_r || pl.copy_meas) {
        void *dst = ws + pl.off_meas;
        e = meas_r ? launch_stage_meas(meas_r, meas_i, A, F, pl.fp, pl.var->layout, dst, stream)
                   : launch_stage_meas(p->meas, nullptr, A, F, pl.fp, pl.var->layout, dst, stream);
        meas = dst;
    }
    if (e != cudaSuccess) return MMN_ERR_CUDA;

    FwdParams fp;
    std::memset(&fp, 0, sizeof(fp));
    fp.x_locs = p->x_locs;
    fp.y_locs = p->y_locs;
    fp.z_locs = p->z_locs;
    fp.nx = p->num_x;
    fp.ny = p->num_y;
    fp.nz = p->num_z;
    fp.nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    fp.vox_start = pl.vox_start;
    fp.vox_count = pl.vox_count;
    fp.ant = ant;
    fp.meas = meas;
    fp.num_ant = pl.a_pad;
    fp.fp = pl.fp;
    fp.nsmp = F;
    fp.ant_per_stage = pl.ant_per_stage;
    fp.mono_flag = hdr + 1;
    fp.k0 = 2.0 * kPi / p->wavelength;
    fp.kd = 2.0 * kPi * p->slope / kC;
    fp.t0 = 1.0 / p->wavelength;
    fp.tblk = (double)kBlockF * p->slope / kC;
    fp.tsmp = p->slope / kC;
    fp.ti = p->is_ti_radar ? 0.15 : 0.0;
    fp.num_tiles = pl.tiles;
    fp.num_splits = pl.splits;
    fp.ant_per_split = pl.ant_per_split;
    fp.image = image;
    fp.vote = vote;
    fp.out_r = out_r;
    fp.out_i = out_i;
    fp.partial = reinterpret_cast<float4 *>(ws + pl.off_partial);
    fp.status = hdr;
    if (pl.smem > 48 * 1024)
        cudaFuncSetAttribute(pl.var->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pl.smem);
    e = launch_fwd(*pl.var, fp, pl.smem, stream);
    if (e != cudaSuccess) return MMN_ERR_CUDA;
    if (pl.splits > 1) {
        e = launch_reduce(fp, stream);
        if (e != cudaSuccess) return MMN_ERR_CUDA;
    }
    return MMN_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

bool is_interp(int mode) { return mode == MMN_MODE_INTERP || mode == MMN_MODE_INTERP_FAST; }

// Constants of the interpolated mode's fast form: 1/lambda as the sum of two floats (the
// reference forms its phase from the FP32 wavelength promoted to FP64) and 1/(2 fft_spacing)
// from the correctly rounded FP32 reciprocal.
void set_fast_fields(InterpParams &ip) {
    const double inv = 1.0 / (double)ip.wavelength;
    ip.inv_lambda_hi = (float)inv;
    ip.inv_lambda_lo = (float)(inv - (double)ip.inv_lambda_hi);
    ip.half_inv_fsp = 0.5f * (1.0f / ip.fft_spacing);
}

}  // namespace

extern "C" {

const char *mmn_version(void) { return "mmnorm_b200 0.1.0 (sm_100a)"; }

int mmn_check_device(int dev) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return MMN_ERR_CUDA;
    return (prop.major == 10 && prop.minor == 0) ? MMN_OK : MMN_ERR_UNSUPPORTED;
}

int mmn_num_variants(int32_t mode) {
    int n = 0;
    const FwdVariant *v = fwd_variants(&n);
    int c = 0;
    for (int i = 0; i < n; ++i) c += (v[i].plain == (mode == MMN_MODE_PLAIN));
    return c;
}

int mmn_variant_info(int32_t mode, int32_t idx, int32_t *voxels_per_thread, int32_t *threads) {
    int n = 0;
    const FwdVariant *v = fwd_variants(&n);
    int c = 0;
    for (int i = 0; i < n; ++i) {
        if (v[i].plain != (mode == MMN_MODE_PLAIN)) continue;
        if (c == idx) {
            if (voxels_per_thread) *voxels_per_thread = v[i].t;
            if (threads) *threads = v[i].nt;
            return MMN_OK;
        }
        ++c;
    }
    return MMN_ERR_INVALID_ARGUMENT;
}

int mmn_set_variant(int32_t mode, int32_t idx) {
    if (mode != MMN_MODE_MIXED && mode != MMN_MODE_PLAIN) return MMN_ERR_INVALID_ARGUMENT;
    int n = 0;
    const FwdVariant *v = fwd_variants(&n);
    int c = 0;
    for (int i = 0; i < n; ++i) {
        if (v[i].plain != (mode == MMN_MODE_PLAIN)) continue;
        if (c == idx) {
            g_variant[mode == MMN_MODE_PLAIN ? 1 : 0].store(i);
            return MMN_OK;
        }
        ++c;
    }
    return MMN_ERR_INVALID_ARGUMENT;
}

int mmn_get_variant(int32_t mode) {
    if (mode != MMN_MODE_MIXED && mode != MMN_MODE_PLAIN) return MMN_ERR_INVALID_ARGUMENT;
    int n = 0;
    const FwdVariant *v = fwd_variants(&n);
    const int cur = g_variant[mode == MMN_MODE_PLAIN ? 1 : 0].load();
    int c = 0;
    for (int i = 0; i < n; ++i) {
        if (v[i].plain != (mode == MMN_MODE_PLAIN)) continue;
        if (i == cur) return c;
        ++c;
    }
    return 0;  // the stored index is not of this mode's list: mmn_backproject uses the first
}

const char *mmn_variant_name(int32_t mode, int32_t idx) {
    int n = 0;
    const FwdVariant *v = fwd_variants(&n);
    int c = 0;
    for (int i = 0; i < n; ++i) {
        if (v[i].plain != (mode == MMN_MODE_PLAIN)) continue;
        if (c == idx) return v[i].name;
        ++c;
    }
    return nullptr;
}

size_t mmn_workspace_bytes(const mmn_problem *p, int32_t mode, int32_t want_vote) {
    (void)want_vote;
    if (check_problem(p, mode) != MMN_OK) return 0;
    if (is_interp(mode)) return kStatusBytes;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    FwdPlan pl;
    if (plan_forward(nvox, 0, nvox, p->num_antennas, p->num_samples, mode, aligned16(p->meas),
                     false, &pl) != MMN_OK)
        return 0;
    return pl.total;
}

int mmn_plan_info(const mmn_problem *p, int32_t mode, int32_t *tiles, int32_t *splits,
                  int32_t *ant_per_stage, int32_t *threads, int32_t *voxels_per_thread) {
    int rc = check_problem(p, mode);
    if (rc != MMN_OK) return rc;
    if (is_interp(mode)) return MMN_ERR_INVALID_ARGUMENT;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    FwdPlan pl;
    rc = plan_forward(nvox, 0, nvox, p->num_antennas, p->num_samples, mode, aligned16(p->meas),
                      false, &pl);
    if (rc != MMN_OK) return rc;
    if (tiles) *tiles = pl.tiles;
    if (splits) *splits = pl.splits;
    if (ant_per_stage) *ant_per_stage = pl.ant_per_stage;
    if (threads) *threads = pl.var->nt;
    if (voxels_per_thread) *voxels_per_thread = pl.var->t;
    return MMN_OK;
}

int mmn_plan_launches(const mmn_problem *p, int32_t mode, int32_t *launches) {
    if (!launches) return MMN_ERR_NULL_POINTER;
    int rc = check_problem(p, mode);
    if (rc != MMN_OK) return rc;
    if (is_interp(mode)) return MMN_ERR_INVALID_ARGUMENT;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    FwdPlan pl;
    rc = plan_forward(nvox, 0, nvox, p->num_antennas, p->num_samples, mode, aligned16(p->meas),
                      false, &pl);
    if (rc != MMN_OK) return rc;
    // antenna records, the staging copy (a layout other than the caller's rows, padding,
    // or misaligned rows), the forward kernel, the split reduction
    *launches = 1 + (pl.copy_meas ? 1 : 0) + 1 + (pl.splits > 1 ? 1 : 0);
    return MMN_OK;
}

int mmn_backproject(const mmn_problem *p, int32_t mode, float *image, float *vote,
                    void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    int rc = check_problem(p, mode);
    if (rc != MMN_OK) return rc;
    if (!image) return MMN_ERR_NULL_POINTER;
    if (misaligned(image, 8) || misaligned(vote, 8)) return MMN_ERR_INVALID_ARGUMENT;
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)))
        return MMN_ERR_WORKSPACE;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    if (p->num_antennas == 0) {
        if (cudaMemsetAsync(image, 0, nvox * 8, stream) != cudaSuccess) return MMN_ERR_CUDA;
        if (vote && cudaMemsetAsync(vote, 0, 3 * nvox * 8, stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        return MMN_OK;
    }
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    if (is_interp(mode)) {
        if (workspace_bytes < kStatusBytes) return MMN_ERR_WORKSPACE;
        if (cudaMemsetAsync(ws, 0, 16, stream) != cudaSuccess) return MMN_ERR_CUDA;
        InterpParams ip;
        std::memset(&ip, 0, sizeof(ip));
        ip.x_locs = p->x_locs;
        ip.y_locs = p->y_locs;
        ip.z_locs = p->z_locs;
        ip.nx = p->num_x;
        ip.ny = p->num_y;
        ip.nz = p->num_z;
        ip.num_ant = p->num_antennas;
        ip.num_rx = p->num_rx;
        ip.nbins = p->num_samples;
        ip.ant = p->antenna_locs;
        ip.rxo = p->rx_offsets;
        ip.meas = reinterpret_cast<const float2 *>(p->meas);
        ip.fft_spacing = (float)p->fft_spacing;
        ip.wavelength = (float)p->wavelength;
        ip.is_ti = p->is_ti_radar;
        ip.start = 0;
        ip.count = nvox;
        ip.nvox = nvox;
        ip.image = reinterpret_cast<float2 *>(image);
        ip.vote = reinterpret_cast<float2 *>(vote);
        if (p->pos_offsets) return MMN_ERR_UNSUPPORTED;
        if (mode == MMN_MODE_INTERP_FAST) {
            set_fast_fields(ip);
            return launch_interp_image_fast(ip, stream) == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
        }
        return launch_interp_image(ip, stream) == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
    }
    FwdPlan pl;
    rc = plan_forward(nvox, 0, nvox, p->num_antennas, p->num_samples, mode, aligned16(p->meas),
                      false, &pl);
    if (rc != MMN_OK) return rc;
    if (workspace_bytes < pl.total) return MMN_ERR_WORKSPACE;
    return run_forward(pl, p, nullptr, nullptr, reinterpret_cast<float2 *>(image),
                       reinterpret_cast<float2 *>(vote), nullptr, nullptr, ws, stream);
}

size_t mmn_normals_workspace_bytes(int64_t num_voxels) {
    (void)num_voxels;
    return kStatusBytes;
}

int mmn_normals(int64_t num_voxels, const float *image, const float *vote, float filter_percent,
                float *normals, uint8_t *mask, float *raw, void *workspace,
                size_t workspace_bytes, cudaStream_t stream) {
    if (num_voxels < 1) return MMN_ERR_INVALID_ARGUMENT;
    if (!image || !vote) return MMN_ERR_NULL_POINTER;
    if (!normals && !mask && !raw) return MMN_ERR_NULL_POINTER;
    if (misaligned(image, 8) || misaligned(vote, 8) || misaligned(normals, 4) ||
        misaligned(raw, 4))
        return MMN_ERR_INVALID_ARGUMENT;
    if (!workspace || workspace_bytes < kStatusBytes ||
        (reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)))
        return MMN_ERR_WORKSPACE;
    if (!(filter_percent >= 0.f) || !std::isfinite(filter_percent))
        return MMN_ERR_INVALID_ARGUMENT;
    unsigned int *max_bits = reinterpret_cast<unsigned int *>(
        static_cast<unsigned char *>(workspace) + 8);
    cudaError_t e = launch_normals(num_voxels, reinterpret_cast<const float2 *>(image),
                                   reinterpret_cast<const float2 *>(vote), filter_percent,
                                   normals, mask, raw, max_bits, stream);
    return e == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

int mmn_image_max_abs(int64_t num_voxels, const float *image, float *max_abs,
                      cudaStream_t stream) {
    if (num_voxels < 1) return MMN_ERR_INVALID_ARGUMENT;
    if (!image || !max_abs) return MMN_ERR_NULL_POINTER;
    if (misaligned(image, 8) || misaligned(max_abs, 4)) return MMN_ERR_INVALID_ARGUMENT;
    // |I| >= 0, so the float's bit pattern orders like the value: atomicMax on the bits
    cudaError_t e = launch_max_abs(num_voxels, reinterpret_cast<const float2 *>(image),
                                   reinterpret_cast<unsigned int *>(max_abs), stream);
    return e == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

int mmn_normals_from_max(int64_t num_voxels, const float *image, const float *vote,
                         const float *max_abs, float filter_percent, float *normals,
                         uint8_t *mask, float *raw, cudaStream_t stream) {
    if (num_voxels < 1) return MMN_ERR_INVALID_ARGUMENT;
    if (!image || !vote || !max_abs) return MMN_ERR_NULL_POINTER;
    if (!normals && !mask && !raw) return MMN_ERR_NULL_POINTER;
    if (misaligned(image, 8) || misaligned(vote, 8) || misaligned(max_abs, 4) ||
        misaligned(normals, 4) || misaligned(raw, 4))
        return MMN_ERR_INVALID_ARGUMENT;
    if (!(filter_percent >= 0.f) || !std::isfinite(filter_percent))
        return MMN_ERR_INVALID_ARGUMENT;
    cudaError_t e = launch_normals_from_max(
        num_voxels, reinterpret_cast<const float2 *>(image),
        reinterpret_cast<const float2 *>(vote), filter_percent, normals, mask, raw,
        reinterpret_cast<const unsigned int *>(max_abs), stream);
    return e == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

size_t mmn_cuda_image_workspace_bytes(int num_antennas, int samples_per_meas,
                                      int use_interpolated_processing) {
    if (use_interpolated_processing) return kStatusBytes;
    if (num_antennas < 0 || samples_per_meas < 1) return 0;
    const int fp = (samples_per_meas + kBlockF - 1) / kBlockF * kBlockF;
    // header + antenna records + interleaved rows; the partial sums are sized per call
    // by the launch extent, so report the bound for the largest split count (64) of a
    // 2^17-voxel launch plus the grid-independent part.  Callers that launch more
    // voxels should query with mmn_cuda_image_workspace_bytes_for.
    return align_up(kStatusBytes) + align_up((size_t)num_antennas * sizeof(AntRec)) +
           align_up((size_t)num_antennas * fp * 16);
}

size_t mmn_cuda_image_workspace_bytes_for(int num_x, int num_y, int num_z, int num_antennas,
                                          int samples_per_meas, int start_ind, int voxel_count,
                                          int use_interpolated_processing) {
    if (use_interpolated_processing) return kStatusBytes;
    const int64_t nvox = (int64_t)num_x * num_y * num_z;
    if (nvox < 1 || num_antennas < 0 || samples_per_meas < 1 || start_ind < 0) return 0;
    int64_t count = voxel_count < 0 ? nvox - start_ind : voxel_count;
    count = std::min<int64_t>(count, nvox - start_ind);
    if (count < 1) return kStatusBytes;
    FwdPlan pl;
    if (plan_forward(nvox, start_ind, count, num_antennas, samples_per_meas, MMN_MODE_MIXED,
                     false, false, &pl) != MMN_OK)
        return 0;
    return pl.total;  // SoA input: plan_forward with meas_aligned=false always stages
}

int mmn_cuda_image(float *p_xyz_r, float *p_xyz_i, const float *x_locs, const float *y_locs,
                   const float *z_locs, const float *antenna_locs, const float *meas_r,
                   const float *meas_i, const float *rx_offsets, float slope, float wavelength,
                   float fft_spacing, int num_x, int num_y, int num_z, int num_antennas,
                   int num_rx_antennas, int samples_per_meas, int start_ind, int is_ti_radar,
                   int use_interpolated_processing, int voxel_count, void *workspace,
                   size_t workspace_bytes, cudaStream_t stream) {
    if (!p_xyz_r || !p_xyz_i || !x_locs || !y_locs || !z_locs) return MMN_ERR_NULL_POINTER;
    if (num_x < 1 || num_y < 1 || num_z < 1 || num_antennas < 0 || num_rx_antennas < 1 ||
        samples_per_meas < 1 || start_ind < 0)
        return MMN_ERR_INVALID_ARGUMENT;
    if (num_antennas > 0 && (!antenna_locs || !meas_r || !meas_i || !rx_offsets))
        return MMN_ERR_NULL_POINTER;
    if (any_misaligned4({p_xyz_r, p_xyz_i, x_locs, y_locs, z_locs, antenna_locs, meas_r,
                         meas_i, rx_offsets}))
        return MMN_ERR_INVALID_ARGUMENT;
    if (!(wavelength > 0.f)) return MMN_ERR_INVALID_ARGUMENT;
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)))
        return MMN_ERR_WORKSPACE;
    const int64_t nvox = (int64_t)num_x * num_y * num_z;
    if (start_ind >= nvox) return MMN_OK;
    int64_t count = voxel_count < 0 ? nvox - start_ind : voxel_count;
    count = std::min<int64_t>(count, nvox - start_ind);
    if (count < 1) return MMN_OK;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    if (num_antennas == 0) {
        if (cudaMemsetAsync(p_xyz_r + start_ind, 0, count * 4, stream) != cudaSuccess ||
            cudaMemsetAsync(p_xyz_i + start_ind, 0, count * 4, stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        return MMN_OK;
    }
    if (use_interpolated_processing) {
        if (workspace_bytes < kStatusBytes) return MMN_ERR_WORKSPACE;
        if (!(fft_spacing > 0.f)) return MMN_ERR_INVALID_ARGUMENT;
        InterpParams ip;
        std::memset(&ip, 0, sizeof(ip));
        ip.x_locs = x_locs;
        ip.y_locs = y_locs;
        ip.z_locs = z_locs;
        ip.nx = num_x;
        ip.ny = num_y;
        ip.nz = num_z;
        ip.num_ant = num_antennas;
        ip.num_rx = num_rx_antennas;
        ip.nbins = samples_per_meas;
        ip.ant = antenna_locs;
        ip.rxo = rx_offsets;
        ip.meas_r = meas_r;
        ip.meas_i = meas_i;
        ip.fft_spacing = fft_spacing;
        ip.wavelength = wavelength;
        ip.is_ti = is_ti_radar;
        ip.start = start_ind;
        ip.count = count;
        ip.nvox = nvox;
        ip.out_r = p_xyz_r;
        ip.out_i = p_xyz_i;
        if (use_interpolated_processing == 2) {
            if (samples_per_meas > kMaxFastBins) return MMN_ERR_TOO_LARGE;
            set_fast_fields(ip);
            return launch_interp_image_fast(ip, stream) == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
        }
        return launch_interp_image(ip, stream) == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
    }
    mmn_problem p;
    std::memset(&p, 0, sizeof(p));
    p.num_x = num_x;
    p.num_y = num_y;
    p.num_z = num_z;
    p.x_locs = x_locs;
    p.y_locs = y_locs;
    p.z_locs = z_locs;
    p.num_antennas = num_antennas;
    p.num_rx = num_rx_antennas;
    p.antenna_locs = antenna_locs;
    p.rx_offsets = rx_offsets;
    p.num_samples = samples_per_meas;
    p.wavelength = (double)wavelength;
    p.slope = (double)slope;
    p.is_ti_radar = is_ti_radar;
    FwdPlan pl;
    int rc = plan_forward(nvox, start_ind, count, num_antennas, samples_per_meas, MMN_MODE_MIXED,
                          false, false, &pl);
    if (rc != MMN_OK) return rc;
    if (workspace_bytes < pl.total) return MMN_ERR_WORKSPACE;
    return run_forward(pl, &p, meas_r, meas_i, nullptr, nullptr, p_xyz_r, p_xyz_i, ws, stream);
}

size_t mmn_cuda_sn_est_workspace_bytes(int num_antennas, int samples_per_meas) {
    (void)num_antennas;
    (void)samples_per_meas;
    return kStatusBytes;
}

}  // extern "C"

namespace {
int cuda_sn_est_impl(bool fast, float *normals_x, float *normals_y, float *normals_z,
                     const int *valid_idx_x, const int *valid_idx_y, const int *valid_idx_z,
                     const float *p_xyz_r, const float *p_xyz_i, const float *x_locs,
                     const float *y_locs, const float *z_locs, const float *antenna_locs,
                     const float *meas_r, const float *meas_i, const float *rx_offsets,
                     float slope, float wavelength, float fft_spacing, int num_x, int num_y,
                     int num_z, int num_antennas, int num_rx_antennas, int num_valid_idx,
                     int samples_per_meas, int start_ind, int is_ti_radar, int count,
                     void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    (void)slope;
    (void)workspace;
    (void)workspace_bytes;
    if (num_valid_idx < 0 || num_x < 1 || num_y < 1 || num_z < 1 || num_antennas < 0 ||
        num_rx_antennas < 1 || samples_per_meas < 1 || start_ind < 0)
        return MMN_ERR_INVALID_ARGUMENT;
    if (num_valid_idx == 0 || start_ind >= num_valid_idx) return MMN_OK;
    if (!normals_x || !normals_y || !normals_z || !valid_idx_x || !valid_idx_y ||
        !valid_idx_z || !p_xyz_r || !p_xyz_i || !x_locs || !y_locs || !z_locs)
        return MMN_ERR_NULL_POINTER;
    if (num_antennas > 0 && (!antenna_locs || !meas_r || !meas_i || !rx_offsets))
        return MMN_ERR_NULL_POINTER;
    if (any_misaligned4({normals_x, normals_y, normals_z, valid_idx_x, valid_idx_y,
                         valid_idx_z, p_xyz_r, p_xyz_i, x_locs, y_locs, z_locs, antenna_locs,
                         meas_r, meas_i, rx_offsets}))
        return MMN_ERR_INVALID_ARGUMENT;
    if (!(wavelength > 0.f) || !(fft_spacing > 0.f)) return MMN_ERR_INVALID_ARGUMENT;
    int64_t n = count < 0 ? (int64_t)num_valid_idx - start_ind : count;
    n = std::min<int64_t>(n, (int64_t)num_valid_idx - start_ind);
    InterpParams ip;
    std::memset(&ip, 0, sizeof(ip));
    ip.x_locs = x_locs;
    ip.y_locs = y_locs;
    ip.z_locs = z_locs;
    ip.nx = num_x;
    ip.ny = num_y;
    ip.nz = num_z;
    ip.num_ant = num_antennas;
    ip.num_rx = num_rx_antennas;
    ip.nbins = samples_per_meas;
    ip.ant = antenna_locs;
    ip.rxo = rx_offsets;
    ip.meas_r = meas_r;
    ip.meas_i = meas_i;
    ip.fft_spacing = fft_spacing;
    ip.wavelength = wavelength;
    ip.is_ti = is_ti_radar;
    ip.start = start_ind;
    ip.count = n;
    ip.vidx_x = valid_idx_x;
    ip.vidx_y = valid_idx_y;
    ip.vidx_z = valid_idx_z;
    ip.img_r = p_xyz_r;
    ip.img_i = p_xyz_i;
    ip.n_x = normals_x;
    ip.n_y = normals_y;
    ip.n_z = normals_z;
    ip.num_valid = num_valid_idx;
    if (fast) {
        if (samples_per_meas > kMaxFastBins) return MMN_ERR_TOO_LARGE;
        set_fast_fields(ip);
        return launch_interp_normals_fast(ip, stream) == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
    }
    return launch_interp_normals(ip, stream) == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}
}  // namespace

extern "C" {

int mmn_cuda_sn_est(float *normals_x, float *normals_y, float *normals_z, const int *valid_idx_x,
                    const int *valid_idx_y, const int *valid_idx_z, const float *p_xyz_r,
                    const float *p_xyz_i, const float *x_locs, const float *y_locs,
                    const float *z_locs, const float *antenna_locs, const float *meas_r,
                    const float *meas_i, const float *rx_offsets, float slope, float wavelength,
                    float fft_spacing, int num_x, int num_y, int num_z, int num_antennas,
                    int num_rx_antennas, int num_valid_idx, int samples_per_meas, int start_ind,
                    int is_ti_radar, int count, void *workspace, size_t workspace_bytes,
                    cudaStream_t stream) {
    return cuda_sn_est_impl(false, normals_x, normals_y, normals_z, valid_idx_x, valid_idx_y,
                            valid_idx_z, p_xyz_r, p_xyz_i, x_locs, y_locs, z_locs, antenna_locs,
                            meas_r, meas_i, rx_offsets, slope, wavelength, fft_spacing, num_x,
                            num_y, num_z, num_antennas, num_rx_antennas, num_valid_idx,
                            samples_per_meas, start_ind, is_ti_radar, count, workspace,
                            workspace_bytes, stream);
}

int mmn_cuda_sn_est_fast(float *normals_x, float *normals_y, float *normals_z,
                         const int *valid_idx_x, const int *valid_idx_y, const int *valid_idx_z,
                         const float *p_xyz_r, const float *p_xyz_i, const float *x_locs,
                         const float *y_locs, const float *z_locs, const float *antenna_locs,
                         const float *meas_r, const float *meas_i, const float *rx_offsets,
                         float slope, float wavelength, float fft_spacing, int num_x, int num_y,
                         int num_z, int num_antennas, int num_rx_antennas, int num_valid_idx,
                         int samples_per_meas, int start_ind, int is_ti_radar, int count,
                         void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    return cuda_sn_est_impl(true, normals_x, normals_y, normals_z, valid_idx_x, valid_idx_y,
                            valid_idx_z, p_xyz_r, p_xyz_i, x_locs, y_locs, z_locs, antenna_locs,
                            meas_r, meas_i, rx_offsets, slope, wavelength, fft_spacing, num_x,
                            num_y, num_z, num_antennas, num_rx_antennas, num_valid_idx,
                            samples_per_meas, start_ind, is_ti_radar, count, workspace,
                            workspace_bytes, stream);
}

int mmn_read_status(void *workspace, int32_t *status, cudaStream_t stream) {
    if (!workspace || !status) return MMN_ERR_NULL_POINTER;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return MMN_ERR_CUDA;
    int32_t s = 0;
    if (cudaMemcpy(&s, workspace, sizeof(s), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MMN_ERR_CUDA;
    *status = s;
    if (cudaMemset(workspace, 0, sizeof(s)) != cudaSuccess) return MMN_ERR_CUDA;
    return MMN_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// Backward pass (adjoint) of the mixed-precision fused backprojection.
// ---------------------------------------------------------------------------------
namespace {

std::atomic<int> g_bwd_variant{0};
std::atomic<int> g_pos_form{MMN_PASS_INTERP};
std::atomic<int> g_pos_variant{0};
std::atomic<int> g_meas_form{MMN_PASS_INTERP};

struct BwdPlan {
    int fp, ant_per_stage, tiles, splits, ant_per_split, threads, vpt;
    size_t smem;
    size_t off_ant, off_meas, off_vox, off_pos, off_mpart, off_nutab, off_nvox, off_npart, total;
    int meas_splits;
    int64_t vox_per_split;
    const void *fn;
    bool nufft;       // position pass in interpolation form
    bool meas_nufft;  // measurement pass in interpolation form
    int nu_n, row;
    int mrow, mranges;
    int64_t mvox_per_range;
};

// image_only: the loss has no vote term (grad_vote NULL): the Horner form needs one chain
// per voxel-antenna and runs the voxel-pair kernel; the interpolation form skips the vote
// terms.  form / meas_form: MMN_PASS_INTERP for the position / measurement pass (used when
// one staged grid row fits a shared-memory stage, i.e. F up to about 1500) or MMN_PASS_HORNER.
int plan_backward(const mmn_problem *p, bool image_only, int form, int meas_form,
                  BwdPlan *pl) {
    const int A = p->num_antennas;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    pl->fp = (p->num_samples + kBlockF - 1) / kBlockF * kBlockF;
    if (pl->fp > kMaxFp) return MMN_ERR_TOO_LARGE;
    pl->nu_n = 2 * p->num_samples;
    const bool nu_fits = (int)sizeof(AntRec) + nufft_row(pl->nu_n) * 16 <= kMaxStageBytes;
    pl->nufft = form == MMN_PASS_INTERP && nu_fits;
    pl->meas_nufft = meas_form == MMN_PASS_INTERP && nu_fits;
    int cap = kMaxStageBytes;
    if (pl->nufft) {
        pl->fn = bwd_pos_nufft_kernel_ptr(g_pos_variant.load(), !image_only, &pl->threads,
                                          &pl->vpt, &cap);
        pl->row = nufft_row(pl->nu_n);
    } else {
        pl->fn = image_only ? bwd_pos_img_kernel_ptr(&pl->threads, &pl->vpt)
                            : bwd_pos_kernel_ptr(g_bwd_variant.load(), &pl->threads, &pl->vpt);
        pl->row = pl->fp;
    }
    const int rec = (int)sizeof(AntRec) + pl->row * 16;
    pl->ant_per_stage = std::max(1, std::min(16, cap / rec));
    pl->smem = 128 + 2 * (size_t)pl->ant_per_stage * rec +
               (size_t)(pl->threads / 32) * pl->ant_per_stage * 3 * sizeof(float);
    const int64_t per_tile = (int64_t)pl->threads * pl->vpt;
    const int64_t tiles = (nvox + per_tile - 1) / per_tile;
    if (tiles > (int64_t)1 << 30) return MMN_ERR_TOO_LARGE;
    pl->tiles = (int)std::max<int64_t>(1, tiles);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (pl->smem > 48 * 1024)
        cudaFuncSetAttribute(pl->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl->smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pl->fn, pl->threads, pl->smem) !=
            cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int64_t slots = (int64_t)sms * per_sm;
    int best_s = 1;
    double best_cost = 1e300;
    const int max_s = std::max(1, std::min(64, (A + pl->ant_per_stage - 1) / pl->ant_per_stage));
    for (int s = 1; s <= max_s; ++s) {
        const int64_t ctas = (int64_t)pl->tiles * s;
        const double waves = (double)((ctas + slots - 1) / slots);
        const double cost = waves * std::ceil((double)A / s) * (1.0 + 0.02 * (s - 1));
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best_s = s;
        }
        if (ctas >= 8 * slots) break;
    }
    int aps = (A + best_s - 1) / best_s;
    aps = (aps + pl->ant_per_stage - 1) / pl->ant_per_stage * pl->ant_per_stage;
    pl->ant_per_split = std::max(aps, 1);
    pl->splits = std::max(1, (A + pl->ant_per_split - 1) / pl->ant_per_split);
    size_t off = kStatusBytes;
    pl->off_ant = off;
    off = align_up(off + (size_t)A * sizeof(AntRec));
    pl->off_meas = off;
    off = align_up(off + (size_t)A * pl->row * 16);
    pl->off_nutab = off;  // interpolation form: twiddles [N] double2, then 1/phihat [F] doubles
    if (pl->nufft || pl->meas_nufft)
        off = align_up(off + (size_t)p->num_samples * sizeof(double) +
                       (size_t)pl->nu_n * sizeof(double2));
    pl->off_nvox = pl->off_npart = off;
    if (pl->meas_nufft) {
        // voxel ranges: enough (antenna group, range) CTAs for two waves
        pl->mrow = pl->nu_n + 16;
        const size_t msmem = nufft_meas_smem(pl->mrow);
        const void *mfn = nufft_meas_kernel_ptr();
        if (msmem > 48 * 1024)
            cudaFuncSetAttribute(mfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem);
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mfn, nufft_meas_warps() * 32,
                                                          msmem) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        const int64_t groups = (A + nufft_meas_warps() - 1) / nufft_meas_warps();
        const int64_t want = (2 * (int64_t)sms * per_sm + groups - 1) / std::max<int64_t>(groups, 1);
        const int64_t chunks = std::max<int64_t>(1, (nvox + 31) / 32);
        const int64_t ranges = std::max<int64_t>(1, std::min<int64_t>({want, 64, chunks}));
        pl->mvox_per_range = (chunks + ranges - 1) / ranges * 32;
        pl->mranges = (int)std::max<int64_t>(1, (nvox + pl->mvox_per_range - 1) / pl->mvox_per_range);
        off = align_up(off + (size_t)nvox * 5 * sizeof(float4));
        pl->off_npart = off;
        off = align_up(off + (size_t)pl->mranges * A * pl->mrow * sizeof(float2));
    }
    pl->off_vox = off;
    off = align_up(off + (size_t)nvox * 3 * sizeof(float4));
    pl->off_pos = off;
    off = align_up(off + (size_t)pl->tiles * A * 3 * sizeof(float));
    pl->meas_splits = bwd_meas_splits(A, pl->fp, nvox);
    const int64_t chunks = (nvox + 511) / 512;
    pl->vox_per_split = (chunks + pl->meas_splits - 1) / pl->meas_splits * 512;
    pl->meas_splits = (int)((nvox + pl->vox_per_split - 1) / pl->vox_per_split);
    pl->off_mpart = off;
    if (pl->meas_splits > 1)
        off = align_up(off + (size_t)pl->meas_splits * A * p->num_samples * sizeof(float2));
    pl->total = off;
    return MMN_OK;
}

}  // namespace

extern "C" size_t mmn_backward_workspace_bytes(const mmn_problem *p) {
    if (check_problem(p, MMN_MODE_MIXED) != MMN_OK) return 0;
    size_t total = 0;
    for (int form = 0; form < 2; ++form) {
        for (int mform = 0; mform < 2; ++mform) {
            BwdPlan pl, pl_img;
            if (plan_backward(p, false, form, mform, &pl) != MMN_OK) return 0;
            if (plan_backward(p, true, form, mform, &pl_img) != MMN_OK) return 0;
            total = std::max(total, std::max(pl.total, pl_img.total));
        }
    }
    return total;
}

// ---------------------------------------------------------------------------------
// Forward in interpolation form: the per-(voxel, antenna) sample sum by an 8-tap gather
// from each antenna's 2x oversampled grid (the position pass's machinery).
// ---------------------------------------------------------------------------------
namespace {

struct NuFwdPlan {
    int n, row, threads, vpt, ant_per_stage, tiles, splits, ant_per_split;
    size_t smem, off_ant, off_rows, off_tab, off_part, total;
    const void *fn;
};

int plan_nufft_forward(const mmn_problem *p, NuFwdPlan *pl) {
    const int A = p->num_antennas, F = p->num_samples;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    pl->n = 2 * F;
    pl->row = nufft_row_fwd(pl->n);  // even: rows of 16-byte multiples
    const int rec = (int)sizeof(AntRec) + pl->row * 8;  // (G.re, G.im) cells
    if (rec > kMaxStageBytes) return MMN_ERR_TOO_LARGE;
    if ((pl->row * 8) % 16 != 0) return MMN_ERR_UNSUPPORTED;  // bulk copies need 16 B rows
    pl->fn = fwd_nufft_kernel_ptr(&pl->threads, &pl->vpt);
    pl->ant_per_stage = std::max(1, std::min(16, 24 * 1024 / rec));
    pl->smem = 128 + 2 * (size_t)pl->ant_per_stage * rec;
    const int64_t per_tile = (int64_t)pl->threads * pl->vpt;
    const int64_t tiles = (nvox + per_tile - 1) / per_tile;
    if (tiles > (int64_t)1 << 30) return MMN_ERR_TOO_LARGE;
    pl->tiles = (int)std::max<int64_t>(1, tiles);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (pl->smem > 48 * 1024)
        cudaFuncSetAttribute(pl->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl->smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pl->fn, pl->threads, pl->smem) !=
            cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int64_t slots = (int64_t)sms * per_sm;
    int best_s = 1;
    double best_cost = 1e300;
    const int max_s = std::max(1, std::min(64, (A + pl->ant_per_stage - 1) / pl->ant_per_stage));
    for (int s = 1; s <= max_s; ++s) {
        const int64_t ctas = (int64_t)pl->tiles * s;
        const double waves = (double)((ctas + slots - 1) / slots);
        const double cost = waves * std::ceil((double)A / s) * (1.0 + 0.02 * (s - 1));
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best_s = s;
        }
        if (ctas >= 8 * slots) break;
    }
    int aps = (A + best_s - 1) / best_s;
    aps = (aps + pl->ant_per_stage - 1) / pl->ant_per_stage * pl->ant_per_stage;
    pl->ant_per_split = std::max(aps, 1);
    pl->splits = std::max(1, (A + pl->ant_per_split - 1) / pl->ant_per_split);
    size_t off = kStatusBytes;
    pl->off_ant = off;
    off = align_up(off + (size_t)A * sizeof(AntRec));
    pl->off_rows = off;
    off = align_up(off + (size_t)A * pl->row * 8);
    pl->off_tab = off;
    off = align_up(off + (size_t)pl->n * sizeof(double2) + (size_t)F * sizeof(double));
    pl->off_part = off;
    if (pl->splits > 1) off = align_up(off + (size_t)pl->splits * nvox * 2 * sizeof(float4));
    pl->total = off;
    return MMN_OK;
}

}  // namespace

extern "C" size_t mmn_backproject_nufft_workspace_bytes(const mmn_problem *p) {
    if (check_problem(p, MMN_MODE_MIXED) != MMN_OK) return 0;
    NuFwdPlan pl;
    return plan_nufft_forward(p, &pl) == MMN_OK ? pl.total : 0;
}

extern "C" int mmn_backproject_nufft(const mmn_problem *p, float *image, float *vote,
                                     void *workspace, size_t workspace_bytes,
                                     cudaStream_t stream) {
    int rc = check_problem(p, MMN_MODE_MIXED);
    if (rc != MMN_OK) return rc;
    if (!image) return MMN_ERR_NULL_POINTER;
    if (misaligned(image, 8) || misaligned(vote, 8)) return MMN_ERR_INVALID_ARGUMENT;
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)))
        return MMN_ERR_WORKSPACE;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    const int A = p->num_antennas, F = p->num_samples;
    if (A == 0) {
        if (cudaMemsetAsync(image, 0, nvox * 8, stream) != cudaSuccess) return MMN_ERR_CUDA;
        if (vote && cudaMemsetAsync(vote, 0, 3 * nvox * 8, stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        return MMN_OK;
    }
    NuFwdPlan pl;
    rc = plan_nufft_forward(p, &pl);
    if (rc != MMN_OK) return rc;
    if (workspace_bytes < pl.total) return MMN_ERR_WORKSPACE;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    if (cudaMemsetAsync(ws, 0, 16, stream) != cudaSuccess) return MMN_ERR_CUDA;
    int32_t *hdr = reinterpret_cast<int32_t *>(ws);
    AntRec *ant = reinterpret_cast<AntRec *>(ws + pl.off_ant);
    if (launch_prep_antennas(p->antenna_locs, p->rx_offsets, p->num_rx, p->pos_offsets, A, A, ant,
                             hdr + 1, stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    const int J0 = F / 2;
    double2 *tw = reinterpret_cast<double2 *>(ws + pl.off_tab);
    double *sc = reinterpret_cast<double *>(tw + pl.n);
    const double k0 = 2.0 * kPi / p->wavelength, kd = 2.0 * kPi * p->slope / kC;
    if (launch_nufft_tables(F, pl.n, J0, sc, tw, stream) != cudaSuccess) return MMN_ERR_CUDA;
    if (launch_nufft_grid(p->meas, A, F, pl.n, J0, k0, kd, sc, tw, ws + pl.off_rows, true,
                          stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    BwdParams bq;
    std::memset(&bq, 0, sizeof(bq));
    FwdParams &f = bq.f;
    f.x_locs = p->x_locs;
    f.y_locs = p->y_locs;
    f.z_locs = p->z_locs;
    f.nx = p->num_x;
    f.ny = p->num_y;
    f.nz = p->num_z;
    f.nvox = nvox;
    f.vox_start = 0;
    f.vox_count = nvox;
    f.ant = ant;
    f.meas = ws + pl.off_rows;
    f.num_ant = A;
    f.fp = pl.row;
    f.ant_per_stage = pl.ant_per_stage;
    f.mono_flag = hdr + 1;
    f.ti = p->is_ti_radar ? 0.15 : 0.0;
    f.num_tiles = pl.tiles;
    f.num_splits = pl.splits;
    f.ant_per_split = pl.ant_per_split;
    f.image = reinterpret_cast<float2 *>(image);
    f.vote = reinterpret_cast<float2 *>(vote);
    f.partial = reinterpret_cast<float4 *>(ws + pl.off_part);
    f.status = hdr;
    bq.nu_n = pl.n;
    bq.nu_u = p->slope / kC;
    bq.nu_k0c = 2.0 * kPi * (1.0 / p->wavelength + (double)J0 * p->slope / kC);
    if (pl.smem > 48 * 1024)
        cudaFuncSetAttribute(pl.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
    void *args[] = {&bq};
    if (cudaLaunchKernel(pl.fn, dim3(pl.tiles * pl.splits), dim3(pl.threads), args, pl.smem,
                         stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    if (pl.splits > 1 && launch_reduce(f, stream) != cudaSuccess) return MMN_ERR_CUDA;
    return MMN_OK;
}

extern "C" int mmn_set_interp_fast_form(int32_t form) {
    if (form < 0 || form > 1) return MMN_ERR_INVALID_ARGUMENT;
    g_interp_fast_form.store(form);
    return MMN_OK;
}

extern "C" int mmn_set_measurement_pass(int32_t form) {
    if (form != MMN_PASS_INTERP && form != MMN_PASS_HORNER) return MMN_ERR_INVALID_ARGUMENT;
    g_meas_form.store(form);
    return MMN_OK;
}

extern "C" int mmn_set_position_pass(int32_t form) {
    if (form != MMN_PASS_INTERP && form != MMN_PASS_HORNER) return MMN_ERR_INVALID_ARGUMENT;
    g_pos_form.store(form);
    return MMN_OK;
}

extern "C" int mmn_num_position_variants(void) { return bwd_pos_nufft_num_variants(); }

extern "C" const char *mmn_position_variant_name(int32_t idx) {
    return bwd_pos_nufft_variant_name(idx);
}

extern "C" int mmn_set_position_variant(int32_t idx) {
    if (idx < 0 || idx >= bwd_pos_nufft_num_variants()) return MMN_ERR_INVALID_ARGUMENT;
    g_pos_variant.store(idx);
    return MMN_OK;
}

extern "C" int mmn_get_position_variant(void) { return g_pos_variant.load(); }

extern "C" int mmn_backproject_backward(const mmn_problem *p, const float *grad_image,
                                        const float *grad_vote, float *grad_meas,
                                        float *grad_pos, void *workspace,
                                        size_t workspace_bytes, cudaStream_t stream) {
    int rc = check_problem(p, MMN_MODE_MIXED);
    if (rc != MMN_OK) return rc;
    if (!grad_meas && !grad_pos) return MMN_ERR_NULL_POINTER;
    if (!grad_image && !grad_vote) return MMN_ERR_NULL_POINTER;
    if (misaligned(grad_image, 8) || misaligned(grad_vote, 8) || misaligned(grad_meas, 8) ||
        misaligned(grad_pos, 4))
        return MMN_ERR_INVALID_ARGUMENT;
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)))
        return MMN_ERR_WORKSPACE;
    const int A = p->num_antennas;
    const int F = p->num_samples;
    if (A == 0) return MMN_OK;
    const bool image_only = grad_vote == nullptr;
    BwdPlan pl;
    rc = plan_backward(p, image_only, g_pos_form.load(), g_meas_form.load(), &pl);
    if (rc != MMN_OK) return rc;
    if (workspace_bytes < pl.total) return MMN_ERR_WORKSPACE;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    if (cudaMemsetAsync(ws, 0, 16, stream) != cudaSuccess) return MMN_ERR_CUDA;
    AntRec *ant = reinterpret_cast<AntRec *>(ws + pl.off_ant);
    int32_t *hdr = reinterpret_cast<int32_t *>(ws);
    if (launch_prep_antennas(p->antenna_locs, p->rx_offsets, p->num_rx, p->pos_offsets, A, A, ant,
                             hdr + 1, stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    BwdParams bp;
    std::memset(&bp, 0, sizeof(bp));
    FwdParams &f = bp.f;
    f.x_locs = p->x_locs;
    f.y_locs = p->y_locs;
    f.z_locs = p->z_locs;
    f.nx = p->num_x;
    f.ny = p->num_y;
    f.nz = p->num_z;
    f.nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    f.vox_start = 0;
    f.vox_count = f.nvox;
    f.ant = ant;
    f.meas = ws + pl.off_meas;
    f.num_ant = A;
    f.fp = pl.fp;
    f.ant_per_stage = pl.ant_per_stage;
    f.mono_flag = hdr + 1;
    f.k0 = 2.0 * kPi / p->wavelength;
    f.kd = 2.0 * kPi * p->slope / kC;
    f.t0 = 1.0 / p->wavelength;
    f.tblk = (double)kBlockF * p->slope / kC;
    f.tsmp = p->slope / kC;
    f.ti = p->is_ti_radar ? 0.15 : 0.0;
    f.num_tiles = pl.tiles;
    f.num_splits = pl.splits;
    f.ant_per_split = pl.ant_per_split;
    f.status = hdr;
    bp.grad_image = reinterpret_cast<const float2 *>(grad_image);
    bp.grad_vote = reinterpret_cast<const float2 *>(grad_vote);
    bp.pos_partial = reinterpret_cast<float *>(ws + pl.off_pos);
    bp.vox_rec = reinterpret_cast<const float4 *>(ws + pl.off_vox);
    bp.grad_meas = reinterpret_cast<float2 *>(grad_meas);
    bp.grad_pos = grad_pos;
    bp.num_samples = F;
    bp.num_ant_real = A;
    bp.num_items = A * (pl.fp / kBlockF);
    bp.meas_splits = pl.meas_splits;
    bp.meas_partial = reinterpret_cast<float2 *>(ws + pl.off_mpart);
    bp.vox_per_split = pl.vox_per_split;
    const int J0 = F / 2;
    double2 *tw = reinterpret_cast<double2 *>(ws + pl.off_nutab);  // 256-aligned
    double *sc = reinterpret_cast<double *>(tw + pl.nu_n);
    if (((grad_pos && pl.nufft) || (grad_meas && pl.meas_nufft)) &&
        launch_nufft_tables(F, pl.nu_n, J0, sc, tw, stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    if (grad_pos && pl.nufft) {
        if (launch_nufft_grid(p->meas, A, F, pl.nu_n, J0, f.k0, f.kd, sc, tw, ws + pl.off_meas,
                              false, stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        BwdParams bq = bp;
        bq.f.fp = pl.row;
        bq.nu_n = pl.nu_n;
        bq.nu_u = p->slope / kC;
        bq.nu_k0c = 2.0 * kPi * (1.0 / p->wavelength + (double)J0 * p->slope / kC);
        if (pl.smem > 48 * 1024)
            cudaFuncSetAttribute(pl.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
        void *args[] = {&bq};
        if (cudaLaunchKernel(pl.fn, dim3(pl.tiles * pl.splits), dim3(pl.threads), args, pl.smem,
                             stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        if (launch_bwd_pos_reduce(bp, stream) != cudaSuccess) return MMN_ERR_CUDA;
    } else if (grad_pos) {
        if (launch_bwd_stage(p->meas, A, F, pl.fp, f.k0, f.kd, image_only ? 1 : 0,
                             ws + pl.off_meas, stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        if (pl.smem > 48 * 1024)
            cudaFuncSetAttribute(pl.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem);
        if (launch_bwd_pos(bp, image_only ? -1 : g_bwd_variant.load(), pl.smem, stream) !=
            cudaSuccess)
            return MMN_ERR_CUDA;
        if (launch_bwd_pos_reduce(bp, stream) != cudaSuccess) return MMN_ERR_CUDA;
    }
    if (grad_meas && pl.meas_nufft) {
        NuMeasParams q;
        std::memset(&q, 0, sizeof(q));
        q.ant = ant;
        q.vox = reinterpret_cast<const float4 *>(ws + pl.off_nvox);
        q.mono_flag = hdr + 1;
        q.part = reinterpret_cast<float2 *>(ws + pl.off_npart);
        q.sc = sc;
        q.tw = tw;
        q.grad_meas = reinterpret_cast<float2 *>(grad_meas);
        q.nvox = f.nvox;
        q.vox_per_range = pl.mvox_per_range;
        q.ti = f.ti;
        q.uq = p->slope / kC;
        q.k0c = 2.0 * kPi * (1.0 / p->wavelength + (double)J0 * p->slope / kC);
        q.num_ant = A;
        q.n = pl.nu_n;
        q.mrow = pl.mrow;
        q.ranges = pl.mranges;
        q.F = F;
        q.J0 = J0;
        if (launch_nufft_meas(q, f, reinterpret_cast<const float2 *>(grad_image),
                              reinterpret_cast<const float2 *>(grad_vote),
                              reinterpret_cast<float4 *>(ws + pl.off_nvox), stream) != cudaSuccess)
            return MMN_ERR_CUDA;
    } else if (grad_meas) {
        if (launch_bwd_vox_rec(bp, reinterpret_cast<float4 *>(ws + pl.off_vox), stream) !=
            cudaSuccess)
            return MMN_ERR_CUDA;
        if (launch_bwd_meas(bp, stream) != cudaSuccess) return MMN_ERR_CUDA;
    }
    return MMN_OK;
}

// ---------------------------------------------------------------------------------
// Backprojection that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they image: hosts that hand
// their whole device pool to another allocator and forbid allocation after start-up,
// plugin hosts that pass only raw device pointers and own every allocation themselves,
// and real-time loops that must not block on the allocator.  mmn_backproject_noalloc
// serves them with a scratch area that is part of the library image itself: a
// file-scope device array, allocated by the CUDA runtime when the library's module is
// loaded into a context and held until the process exits.  Its device address is looked
// up (cudaGetSymbolAddress) on the first call made in each CUDA context, with that
// context current, and cached under the context's unique id -- an address from one
// context is not mapped in another, and a context created after cudaDeviceReset gets a
// new id.  The caller still owns inputs and outputs.
// ---------------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;  // 16 MiB per context
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

typedef CUresult(CUDAAPI *CtxGetCurrentFn)(CUcontext *);
typedef CUresult(CUDAAPI *CtxGetIdFn)(CUcontext, unsigned long long *);

struct NoAllocEntry {
    unsigned long long ctx_id;
    void *addr;
};
std::mutex g_noalloc_mutex;
std::vector<NoAllocEntry> g_noalloc_cache;
bool g_noalloc_fns_looked_up = false;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Unique id of the calling thread's current context; false when no context is current
// or the driver cannot tell (then nothing is cached).  Caller holds g_noalloc_mutex.
bool current_context_id(unsigned long long *id) {
    if (!g_noalloc_fns_looked_up) {
        g_noalloc_fns_looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent",
                                             reinterpret_cast<void **>(&g_ctx_get_current),
                                             12000, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            g_ctx_get_current = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId",
                                             reinterpret_cast<void **>(&g_ctx_get_id), 12000,
                                             cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            g_ctx_get_id = nullptr;
        cudaGetLastError();  // a failed lookup leaves nothing behind for later calls
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of the scratch array in the current context.  In host code the array's
// name only stands in for the symbol, so the address has to come from the runtime.
int noalloc_scratch(void **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    unsigned long long id = 0;
    if (current_context_id(&id)) {
        for (const NoAllocEntry &e : g_noalloc_cache)
            if (e.ctx_id == id) {
                *out = e.addr;
                return MMN_OK;
            }
    }
    // first call in this context (cudaGetSymbolAddress also makes the device's primary
    // context current if no context is)
    void *addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr)
        return MMN_ERR_CUDA;
    if (current_context_id(&id)) g_noalloc_cache.push_back({id, addr});
    *out = addr;
    return MMN_OK;
}

}  // namespace

extern "C" int mmn_noalloc_read_status(int32_t *status, cudaStream_t stream) {
    if (!status) return MMN_ERR_NULL_POINTER;
    void *scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc != MMN_OK) return rc;
    return mmn_read_status(scratch, status, stream);
}

extern "C" int mmn_backproject_noalloc(const mmn_problem *p, int32_t mode, float *image,
                                       float *vote, cudaStream_t stream) {
    int rc = check_problem(p, mode);
    if (rc != MMN_OK) return rc;
    if (!image) return MMN_ERR_NULL_POINTER;
    if (misaligned(image, 8) || misaligned(vote, 8)) return MMN_ERR_INVALID_ARGUMENT;
    const int64_t nvox = (int64_t)p->num_x * p->num_y * p->num_z;
    FwdPlan pl;
    const bool full = !is_interp(mode) && p->num_antennas > 0;
    if (full) {
        rc = plan_forward(nvox, 0, nvox, p->num_antennas, p->num_samples, mode,
                          aligned16(p->meas), false, &pl);
        if (rc != MMN_OK) return rc;
        // every voxel tile takes the whole antenna range: no partial sums to hold
        pl.splits = 1;
        pl.ant_per_split = pl.a_pad;
        pl.total = pl.off_partial;
        if (pl.total > kNoAllocScratchBytes) return MMN_ERR_TOO_LARGE;
    }
    void *scratch = nullptr;
    rc = noalloc_scratch(&scratch);
    if (rc != MMN_OK) return rc;
    if (!full)  // interpolated mode and empty apertures only need the status header
        return mmn_backproject(p, mode, image, vote, scratch, kNoAllocScratchBytes, stream);
    return run_forward(pl, p, nullptr, nullptr, reinterpret_cast<float2 *>(image),
                       reinterpret_cast<float2 *>(vote), nullptr, nullptr,
                       static_cast<unsigned char *>(scratch), stream);
}

// ---------------------------------------------------------------------------------
// Batched persistent launch: many objects (uneven grids, apertures and sample counts)
// in one launch over a cost-sorted (object, voxel tile, antenna split) work list.
// ---------------------------------------------------------------------------------
struct mmn_batch {
    int n = 0;
    int mode = 0;
    const FwdVariant *var = nullptr;
    size_t smem = 0;
    int ctas = 0;
    struct Obj {
        int fp = 0, a_pad = 0, nas = 0, tiles = 0, splits = 1, aps = 0;
        int64_t nvox = 0;
        size_t off_ant = 0, off_meas = 0, off_partial = 0;
    };
    std::vector<mmn_problem> probs;
    std::vector<Obj> obj;
    std::vector<FwdParams> params;  // filled at upload (device pointers into the workspace)
    std::vector<int4> items;
    std::vector<float *> images, votes;
    size_t off_flags = 0, off_counter = 0, off_params = 0, off_items = 0, total = 0;
    void *uploaded_ws = nullptr;
};

extern "C" int mmn_batch_create(const mmn_problem *problems, int32_t num_objects, int32_t mode,
                                float *const *images, float *const *votes,
                                int32_t items_per_slot, mmn_batch **batch,
                                size_t *workspace_bytes) {
    if (!problems || !images || !batch || !workspace_bytes) return MMN_ERR_NULL_POINTER;
    if (num_objects < 1 || mode != MMN_MODE_MIXED) return MMN_ERR_INVALID_ARGUMENT;
    for (int o = 0; o < num_objects; ++o) {
        const int rc = check_problem(&problems[o], mode);
        if (rc != MMN_OK) return rc;
        if (!images[o]) return MMN_ERR_NULL_POINTER;
        if (misaligned(images[o], 8) || (votes && misaligned(votes[o], 8)))
            return MMN_ERR_INVALID_ARGUMENT;
    }
    if (items_per_slot <= 0) items_per_slot = 8;
    int nvar = 0;
    const FwdVariant *vars = fwd_variants(&nvar);
    int vi = variant_index_for(mode);
    if (vi < 0 || vi >= nvar || vars[vi].plain || !vars[vi].persistent_fn) {
        vi = 0;
        while (vi < nvar && (vars[vi].plain || !vars[vi].persistent_fn)) ++vi;
        if (vi >= nvar) return MMN_ERR_UNSUPPORTED;
    }
    mmn_batch *b = new mmn_batch();
    b->n = num_objects;
    b->mode = mode;
    b->var = &vars[vi];
    b->probs.assign(problems, problems + num_objects);
    b->images.assign(images, images + num_objects);
    b->votes.assign(num_objects, nullptr);
    if (votes)
        for (int o = 0; o < num_objects; ++o) b->votes[o] = votes[o];
    b->obj.resize(num_objects);
    const bool pairs = b->var->layout == 2;
    size_t max_stage = 0;
    for (int o = 0; o < num_objects; ++o) {
        auto &ob = b->obj[o];
        const mmn_problem &p = problems[o];
        ob.fp = (p.num_samples + kBlockF - 1) / kBlockF * kBlockF;
        if (ob.fp > kMaxFp) {
            delete b;
            return MMN_ERR_TOO_LARGE;
        }
        ob.a_pad = pairs ? p.num_antennas + (p.num_antennas & 1) : p.num_antennas;
        const int rec = (int)sizeof(AntRec) + ob.fp * b->var->esz;
        const int cap = b->var->max_stage_bytes > 0 ? b->var->max_stage_bytes : kMaxStageBytes;
        ob.nas = std::max(1, std::min(16, cap / rec));
        if (pairs) ob.nas = std::max(2, ob.nas & ~1);
        max_stage = std::max(max_stage, (size_t)ob.nas * rec);
        ob.nvox = (int64_t)p.num_x * p.num_y * p.num_z;
    }
    b->smem = 128 + 2 * max_stage;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (b->smem > 48 * 1024)
        cudaFuncSetAttribute(b->var->persistent_fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)b->smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->var->persistent_fn, b->var->nt,
                                                      b->smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    b->ctas = sms * per_sm;
    // item granularity: about items_per_slot items per resident CTA
    const int64_t tile_vox = (int64_t)b->var->nt * b->var->t;
    double total_cost = 0;
    for (int o = 0; o < num_objects; ++o)
        total_cost += (double)b->obj[o].nvox * b->obj[o].a_pad * b->obj[o].fp;
    const double target = std::max(1.0, total_cost / ((double)b->ctas * items_per_slot));
    std::vector<std::pair<double, int4>> work;
    for (int o = 0; o < num_objects; ++o) {
        auto &ob = b->obj[o];
        ob.tiles = (int)((ob.nvox + tile_vox - 1) / tile_vox);
        if (ob.a_pad == 0) {
            ob.splits = 0;
            continue;
        }
        const double tile_cost = (double)tile_vox * ob.a_pad * ob.fp;
        const int max_s = (ob.a_pad + ob.nas - 1) / ob.nas;
        int s = (int)std::ceil(tile_cost / target);
        s = std::max(1, std::min(s, std::min(max_s, 64)));
        ob.aps = (ob.a_pad + s - 1) / s;
        ob.aps = (ob.aps + ob.nas - 1) / ob.nas * ob.nas;
        ob.splits = (ob.a_pad + ob.aps - 1) / ob.aps;
        for (int t = 0; t < ob.tiles; ++t) {
            const int64_t v = std::min<int64_t>(tile_vox, ob.nvox - (int64_t)t * tile_vox);
            for (int sp = 0; sp < ob.splits; ++sp) {
                const int na = std::min(ob.aps, ob.a_pad - sp * ob.aps);
                work.push_back({(double)v * na * ob.fp, make_int4(o, t, sp, 0)});
            }
        }
    }
    std::stable_sort(work.begin(), work.end(),
                     [](const std::pair<double, int4> &x, const std::pair<double, int4> &y) {
                         return x.first > y.first;
                     });
    b->items.reserve(work.size());
    for (auto &w : work) b->items.push_back(w.second);
    // workspace layout
    size_t off = kStatusBytes;
    b->off_flags = off;
    off = align_up(off + (size_t)num_objects * sizeof(int32_t));
    b->off_counter = off;
    off = align_up(off + sizeof(int));
    b->off_params = off;
    off = align_up(off + (size_t)num_objects * sizeof(FwdParams));
    b->off_items = off;
    off = align_up(off + b->items.size() * sizeof(int4) + 16);
    for (int o = 0; o < num_objects; ++o) {
        auto &ob = b->obj[o];
        const int rows = b->var->layout == 2 ? ob.a_pad / 2 : ob.a_pad;
        const size_t row_bytes = (size_t)ob.fp * (b->var->layout == 2 ? 16 : b->var->esz);
        ob.off_ant = off;
        off = align_up(off + (size_t)ob.a_pad * sizeof(AntRec));
        ob.off_meas = off;
        off = align_up(off + (size_t)rows * row_bytes);
        ob.off_partial = off;
        if (ob.splits > 1) off = align_up(off + (size_t)ob.splits * ob.nvox * 8 * sizeof(float));
    }
    b->total = off;
    *batch = b;
    *workspace_bytes = b->total;
    return MMN_OK;
}

extern "C" int mmn_batch_upload(mmn_batch *b, void *workspace, size_t workspace_bytes,
                                cudaStream_t stream) {
    if (!b || !workspace) return MMN_ERR_NULL_POINTER;
    if ((reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)) || workspace_bytes < b->total)
        return MMN_ERR_WORKSPACE;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    b->params.assign(b->n, FwdParams());
    for (int o = 0; o < b->n; ++o) {
        const mmn_problem &p = b->probs[o];
        const auto &ob = b->obj[o];
        FwdParams &f = b->params[o];
        std::memset(&f, 0, sizeof(f));
        f.x_locs = p.x_locs;
        f.y_locs = p.y_locs;
        f.z_locs = p.z_locs;
        f.nx = p.num_x;
        f.ny = p.num_y;
        f.nz = p.num_z;
        f.nvox = ob.nvox;
        f.vox_start = 0;
        f.vox_count = ob.nvox;
        f.ant = reinterpret_cast<const AntRec *>(ws + ob.off_ant);
        f.meas = ws + ob.off_meas;
        f.num_ant = ob.a_pad;
        f.fp = ob.fp;
        f.nsmp = p.num_samples;
        f.ant_per_stage = ob.nas;
        f.mono_flag = reinterpret_cast<const int32_t *>(ws + b->off_flags) + o;
        f.k0 = 2.0 * kPi / p.wavelength;
        f.kd = 2.0 * kPi * p.slope / kC;
        f.t0 = 1.0 / p.wavelength;
        f.tblk = (double)kBlockF * p.slope / kC;
        f.tsmp = p.slope / kC;
        f.ti = p.is_ti_radar ? 0.15 : 0.0;
        f.num_tiles = ob.tiles;
        f.num_splits = std::max(1, ob.splits);
        f.ant_per_split = ob.aps;
        f.image = reinterpret_cast<float2 *>(b->images[o]);
        f.vote = reinterpret_cast<float2 *>(b->votes[o]);
        f.partial = reinterpret_cast<float4 *>(ws + ob.off_partial);
        f.status = reinterpret_cast<int32_t *>(ws);
    }
    if (cudaMemcpyAsync(ws + b->off_params, b->params.data(), b->n * sizeof(FwdParams),
                        cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    if (!b->items.empty() &&
        cudaMemcpyAsync(ws + b->off_items, b->items.data(), b->items.size() * sizeof(int4),
                        cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return MMN_ERR_CUDA;
    b->uploaded_ws = workspace;
    return MMN_OK;
}

extern "C" int mmn_batch_run(mmn_batch *b, void *workspace, cudaStream_t stream) {
    if (!b || !workspace) return MMN_ERR_NULL_POINTER;
    if (workspace != b->uploaded_ws) return MMN_ERR_WORKSPACE;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    if (cudaMemsetAsync(ws, 0, 16, stream) != cudaSuccess) return MMN_ERR_CUDA;
    if (cudaMemsetAsync(ws + b->off_counter, 0, sizeof(int), stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    for (int o = 0; o < b->n; ++o) {
        const mmn_problem &p = b->probs[o];
        const auto &ob = b->obj[o];
        const int64_t V = ob.nvox;
        if (p.num_antennas == 0) {
            if (cudaMemsetAsync(b->images[o], 0, V * 8, stream) != cudaSuccess) return MMN_ERR_CUDA;
            if (b->votes[o] && cudaMemsetAsync(b->votes[o], 0, 3 * V * 8, stream) != cudaSuccess)
                return MMN_ERR_CUDA;
            continue;
        }
        if (launch_prep_antennas(p.antenna_locs, p.rx_offsets, p.num_rx, p.pos_offsets,
                                 p.num_antennas, ob.a_pad,
                                 reinterpret_cast<AntRec *>(ws + ob.off_ant),
                                 reinterpret_cast<int32_t *>(ws + b->off_flags) + o,
                                 stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        if (launch_stage_meas(p.meas, nullptr, p.num_antennas, p.num_samples, ob.fp,
                              b->var->layout, ws + ob.off_meas, stream) != cudaSuccess)
            return MMN_ERR_CUDA;
    }
    if (!b->items.empty()) {
        BatchParams bp;
        bp.objs = reinterpret_cast<const FwdParams *>(ws + b->off_params);
        bp.items = reinterpret_cast<const int4 *>(ws + b->off_items);
        bp.num_items = (int32_t)b->items.size();
        bp.pad0 = 0;
        bp.counter = reinterpret_cast<int *>(ws + b->off_counter);
        void *args[] = {&bp};
        const int grid = std::min<int>(b->ctas, (int)b->items.size());
        if (cudaLaunchKernel(b->var->persistent_fn, dim3(grid), dim3(b->var->nt), args, b->smem,
                             stream) != cudaSuccess)
            return MMN_ERR_CUDA;
    }
    for (int o = 0; o < b->n; ++o)
        if (b->obj[o].splits > 1 && launch_reduce(b->params[o], stream) != cudaSuccess)
            return MMN_ERR_CUDA;
    return MMN_OK;
}

extern "C" int mmn_batch_info(const mmn_batch *b, int32_t *num_items, int32_t *ctas,
                              int32_t *threads, int32_t *voxels_per_thread) {
    if (!b) return MMN_ERR_NULL_POINTER;
    if (num_items) *num_items = (int32_t)b->items.size();
    if (ctas) *ctas = b->ctas;
    if (threads) *threads = b->var->nt;
    if (voxels_per_thread) *voxels_per_thread = b->var->t;
    return MMN_OK;
}

extern "C" void mmn_batch_destroy(mmn_batch *b) { delete b; }

/*
 * mmnorm_b200.h -- C ABI of the B200 (sm_100a) near-field SAR backprojection and
 * mmWave surface-normal vote.
 *
 * Every pointer argument is a DEVICE pointer unless the name ends in _host.  Every
 * entry point is asynchronous on the given stream, allocates nothing unless stated,
 * and returns MMN_OK or an MMN_ERR_* code; no C++ exception crosses this boundary.
 * Calls on distinct streams with distinct workspaces are thread-safe.
 *
 * Conventions shared with the reference (src/data_processing/cuda/imaging_gpu.cu):
 *   - voxel (x, y, z) has flat index  x*NY*NZ + y*NZ + z                (:121-122)
 *   - virtual antenna i has TX position antenna_locs[i] and RX position
 *     antenna_locs[i] + rx_offsets[i % num_rx]                           (:67-83)
 *   - round-trip distance d = |v - tx| + |v - rx|, plus 0.15 m if is_ti_radar (:86-88)
 *   - full matched filter: sum_j m[i,j] exp(-j 2 pi d (1/wavelength + j slope/c)) (:112)
 *   - interpolated mode: m_fft[i, floor(d/fft_spacing/2)] exp(-j 2 pi d/wavelength),
 *     skipped when d < 0 or d > fft_spacing * num_bins                   (:90-105)
 *   - normal vote: sum_i Re(c_i conj(I))/|I| (tx_i + o_i/2 - v)
 *     (src/data_processing/cuda/surface_normal_est.cu:128-145)
 * Complex arrays are interleaved (re, im) float32 pairs, i.e. complex64.
 */
#ifndef MMNORM_B200_H
#define MMNORM_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MMN_OK 0
#define MMN_ERR_INVALID_ARGUMENT 1 /* bad size, mode, flag or array alignment  */
#define MMN_ERR_NULL_POINTER 2     /* a required pointer is NULL               */
#define MMN_ERR_UNSUPPORTED 3      /* device is not sm_100 / feature missing   */
#define MMN_ERR_WORKSPACE 4        /* workspace NULL, misaligned or too small  */
#define MMN_ERR_CUDA 5             /* a CUDA runtime call failed               */
#define MMN_ERR_TIMEOUT 6          /* a bounded in-kernel wait gave up         */
#define MMN_ERR_TOO_LARGE 7        /* a size exceeds a documented maximum      */

/* forward-projection forms */
#define MMN_MODE_MIXED 0  /* FP64 range + wrap, FP32 rotation recurrence (default)  */
#define MMN_MODE_PLAIN 1  /* FP32 range and phase, one sincosf per sample           */
#define MMN_MODE_INTERP 2 /* reference interpolated mode (range-FFT bin + 1 phasor) */
/* Interpolated mode, fast form (no counterpart in the reference): the reference's FP32
 * path length and range bin, so the same range-FFT sample is gathered, with the phasor
 * exp(-j 2 pi d / lambda) formed from the wrapped FP32 turn count (1/lambda split into two
 * floats) and the hardware sine/cosine instead of FP64 cos and sin: about 5e-7 relative
 * per term from the reference's phasor.  Bins up to 2^22 (else MMN_ERR_TOO_LARGE). */
#define MMN_MODE_INTERP_FAST 3

/* Form of the fast interpolated passes (no reference counterpart), process-wide:
 * 0 (default) two voxels per thread in packed FP32 instructions, 1 the same arithmetic
 * in scalar instructions.  Both give the reference's range bins and path lengths. */
int mmn_set_interp_fast_form(int32_t form);

/* Problem description.  All array pointers are device pointers, aligned to their
 * element: float arrays to 4 bytes, complex64 arrays (samples, images, votes and their
 * gradients) to 8 bytes; any other pointer returns MMN_ERR_INVALID_ARGUMENT before a
 * device call. */
typedef struct mmn_problem {
    int32_t num_x, num_y, num_z;  /* voxel grid                                   */
    const float *x_locs;          /* [num_x] voxel centres along x                */
    const float *y_locs;          /* [num_y]                                      */
    const float *z_locs;          /* [num_z]                                      */
    int32_t num_antennas;         /* virtual antennas A*R (TX repeated per RX)    */
    int32_t num_rx;               /* R >= 1                                       */
    const float *antenna_locs;    /* [num_antennas, 3] TX positions               */
    const float *rx_offsets;      /* [num_rx, 3]                                  */
    const float *pos_offsets;     /* [num_antennas, 3] added to TX and RX, or NULL */
    int32_t num_samples;          /* F samples (full) or range bins (interp)      */
    const float *meas;            /* complex64 [num_antennas, num_samples]        */
    double wavelength;            /* c / start frequency                          */
    double slope;                 /* Hz per sample                                */
    double fft_spacing;           /* interpolated mode only                       */
    int32_t is_ti_radar;          /* add 0.15 m to the round-trip distance        */
    int32_t reserved;
} mmn_problem;

/* Library identification and device check (0 when device `dev` is an sm_100 part). */
const char *mmn_version(void);
int mmn_check_device(int dev);

/* Bytes of device workspace mmn_backproject needs for `p` in `mode` (256-aligned).
 * Returns 0 for an invalid problem.  Depends on the current device (occupancy). */
size_t mmn_workspace_bytes(const mmn_problem *p, int32_t mode, int32_t want_vote);

/* Kernel variants of the full-mode forward pass (voxels per thread x threads per CTA)
 * for the autotuner; no reference counterpart (the reference has one fixed launch,
 * block=512, py_image_gpu.py:272-273).  mmn_set_variant selects the process-wide
 * variant mmn_backproject uses for MMN_MODE_MIXED / MMN_MODE_PLAIN; mmn_get_variant
 * returns the selected index (or MMN_ERR_INVALID_ARGUMENT for another mode). */
int mmn_num_variants(int32_t mode);
int mmn_variant_info(int32_t mode, int32_t idx, int32_t *voxels_per_thread, int32_t *threads);
int mmn_set_variant(int32_t mode, int32_t idx);
int mmn_get_variant(int32_t mode);
const char *mmn_variant_name(int32_t mode, int32_t idx); /* NULL for a bad index */

/* The decomposition mmn_backproject will use for `p`: voxel tiles, antenna splits,
 * antennas per shared-memory stage, threads per CTA, voxels per thread. */
int mmn_plan_info(const mmn_problem *p, int32_t mode, int32_t *tiles, int32_t *splits,
                  int32_t *ant_per_stage, int32_t *threads, int32_t *voxels_per_thread);
/* Kernel launches mmn_backproject makes for `p` in `mode` (full modes): antenna records,
 * the staging copy of the sample rows when the kernel form needs one, the forward kernel,
 * and the split reduction when the antenna range is split.  No reference counterpart. */
int mmn_plan_launches(const mmn_problem *p, int32_t mode, int32_t *launches);

/*
 * Fused backprojection + vote.  image: complex64 [V] raw sum over all virtual
 * antennas and samples (not normalised).  vote (may be NULL): complex64 [3, V], the
 * plane k holding W_k(v) = sum_i c_i(v) * (tx_i + o_i/2 - v)_k, from which the
 * reference's normal is Re(conj(I) W)/|I|.  Replaces the cuda_image launch in
 * src/data_processing/cuda/py_image_gpu.py:189-199 and, for the vote, the
 * cuda_sn_est launch in src/data_processing/cuda/py_sn_est_gpu.py:229-246.
 */
int mmn_backproject(const mmn_problem *p, int32_t mode, float *image, float *vote,
                    void *workspace, size_t workspace_bytes, cudaStream_t stream);

/*
 * Adjoint of mmn_backproject in MMN_MODE_MIXED (no counterpart in the reference, which
 * has no gradients).  Given dL/dI (grad_image, complex64 [V]) and dL/dW (grad_vote,
 * complex64 [3, V]; either may be NULL = zero) in the convention grad = dL/dRe + i dL/dIm,
 * writes dL/dmeas (grad_meas, complex64 [num_antennas, num_samples], or NULL) and the
 * gradient with respect to per-antenna position offsets added to TX and RX (grad_pos,
 * float32 [num_antennas, 3], or NULL).  Phasors are recomputed; nothing per
 * (voxel, antenna) is stored.  Needs mmn_backward_workspace_bytes() of workspace.
 */
size_t mmn_backward_workspace_bytes(const mmn_problem *p);
int mmn_backproject_backward(const mmn_problem *p, const float *grad_image,
                             const float *grad_vote, float *grad_meas, float *grad_pos,
                             void *workspace, size_t workspace_bytes, cudaStream_t stream);

/*
 * How the backward evaluates the two per-(voxel, antenna) sample sums the position
 * gradient needs (no reference counterpart).  MMN_POS_INTERP (the default): interpolation
 * with an 8-cell exponential-of-semicircle kernel from each antenna's spectrum on a 2x
 * oversampled grid (a type-2 non-uniform FFT; ~1e-7 relative, the FP32 chains' level),
 * used when F <= ~1500; MMN_POS_HORNER: two FP32 Horner chains over all F samples, as the
 * forward evaluates its sum.  Process-wide; the measurement gradient is the same in both.
 */
#define MMN_PASS_INTERP 0
#define MMN_PASS_HORNER 1
#define MMN_POS_INTERP MMN_PASS_INTERP
#define MMN_POS_HORNER MMN_PASS_HORNER
int mmn_set_position_pass(int32_t form);
/*
 * The same choice for the measurement gradient dL/dm[a,j] = sum_v G conj(p) (no reference
 * counterpart): MMN_PASS_INTERP (the default) spreads each voxel onto 8 cells of the
 * antenna's oversampled grid and transforms each grid back to the F samples (type-1
 * non-uniform FFT, deterministic warp reductions; F up to ~1500); MMN_PASS_HORNER sums
 * over voxels for every sample.  Process-wide.
 */
int mmn_set_measurement_pass(int32_t form);
/* Launch shapes of the interpolation form (voxels per thread, threads, stage size) for the
 * autotuner; process-wide, like mmn_set_variant. */
int mmn_num_position_variants(void);
const char *mmn_position_variant_name(int32_t idx); /* NULL for a bad index */
int mmn_set_position_variant(int32_t idx);
int mmn_get_position_variant(void); /* the selected index */

/*
 * Fused backprojection + vote with the per-(voxel, antenna) sample sum evaluated by
 * interpolation (no counterpart in the reference; not its "interpolated mode", which reads
 * one range bin): each antenna's samples go once onto a 2x oversampled grid, and each
 * (voxel, antenna) gathers 8 cells with exponential-of-semicircle weights -- a type-2
 * non-uniform FFT, O(8) per pair instead of O(F).  Same outputs and problem fields as
 * mmn_backproject in MMN_MODE_MIXED, ~1e-7 relative from it; F up to ~1500
 * (MMN_ERR_TOO_LARGE above).  Needs mmn_backproject_nufft_workspace_bytes() of workspace.
 */
size_t mmn_backproject_nufft_workspace_bytes(const mmn_problem *p);
int mmn_backproject_nufft(const mmn_problem *p, float *image, float *vote, void *workspace,
                          size_t workspace_bytes, cudaStream_t stream);

/*
 * Batched persistent launch (no counterpart in the reference, which images one object per
 * call; mmwave_reconstruction.sh:61-69 loops over objects in the shell).  Many objects --
 * each its own voxel grid, aperture, sample count and radar constants -- run in ONE
 * persistent kernel launch over a work list of (object, voxel tile, antenna split) items
 * sorted by cost, largest first; CTAs pop items from a global counter.  MMN_MODE_MIXED only.
 *   mmn_batch_create: plans the work list (about items_per_slot items per resident CTA;
 *     <= 0 picks 8) for the given problems and output buffers (images[o]: complex64 [V_o];
 *     votes[o]: complex64 [3, V_o] or NULL; votes itself may be NULL); returns the
 *     workspace size.  Host-side only.
 *   mmn_batch_upload: writes the plan's tables into the workspace (synchronises `stream`).
 *   mmn_batch_run: per-object preparation kernels, the persistent kernel and the split
 *     reductions -- only kernel launches and memsets, so it can be captured in a CUDA graph.
 * Each object's result equals mmn_backproject's up to summation order across antenna splits.
 */
typedef struct mmn_batch mmn_batch;
int mmn_batch_create(const mmn_problem *problems, int32_t num_objects, int32_t mode,
                     float *const *images, float *const *votes, int32_t items_per_slot,
                     mmn_batch **batch, size_t *workspace_bytes);
int mmn_batch_upload(mmn_batch *batch, void *workspace, size_t workspace_bytes,
                     cudaStream_t stream);
int mmn_batch_run(mmn_batch *batch, void *workspace, cudaStream_t stream);
int mmn_batch_info(const mmn_batch *batch, int32_t *num_items, int32_t *ctas, int32_t *threads,
                   int32_t *voxels_per_thread);
void mmn_batch_destroy(mmn_batch *batch);

/*
 * mmn_backproject without any device allocation (no counterpart in the reference, which
 * allocates through pycuda on every call).  For callers that cannot call cudaMalloc
 * where they image -- a host that hands its whole device pool to its own allocator and
 * forbids allocation after start-up, a plugin host that passes only raw device pointers,
 * a real-time loop that must not block on the allocator.  Same inputs, outputs and modes
 * as mmn_backproject; the scratch comes from a 16 MiB device array built into the
 * library, which every GPU (every CUDA context) that loads the library holds until the
 * process exits.
 *   - Limit: the antenna records plus the staged samples must fit 16 MiB: 256 + 64*A
 *     bytes, plus 8*A*roundup(F, 32) when the default form stages the rows (F not a
 *     multiple of 32, or rows not 16-byte aligned; 16 bytes per sample in the first-order
 *     voxel-pair variants), e.g. A*F up to about two million antenna-samples when staged;
 *     larger problems return MMN_ERR_TOO_LARGE before anything runs.  Every voxel tile takes the whole antenna range (no antenna split),
 *     so problems with few voxels run slower than through mmn_backproject.
 *   - The array's device address belongs to a CUDA context.  The first call in each
 *     context (normally the device's primary context) looks it up with
 *     cudaGetSymbolAddress, with that context current, and caches it under the context's
 *     unique id; make that first call before any stream capture.
 *   - All calls in a context share the one array and each call re-initialises what it
 *     reads; calls whose work overlaps on the GPU (different streams, or host threads
 *     without ordering) race on it and must be serialised by the caller.
 *   - The array starts with the status word of its bounded in-kernel waits: read and
 *     clear it with mmn_noalloc_read_status (MMN_ERR_TIMEOUT there means the last call's
 *     image and vote are not valid).  The next call clears it.
 */
int mmn_backproject_noalloc(const mmn_problem *p, int32_t mode, float *image, float *vote,
                            cudaStream_t stream);

/*
 * Status word of mmn_backproject_noalloc's built-in scratch array in the current context
 * (mmn_read_status for that array): synchronises `stream`, copies the word to *status and
 * clears it.  MMN_OK in *status after a completed call; MMN_ERR_TIMEOUT if a bounded wait
 * gave up.
 */
int mmn_noalloc_read_status(int32_t *status, cudaStream_t stream);

/*
 * Unit surface normals from (image, vote): mask |I| > filter_percent * max|I|
 * (src/data_processing/cuda/py_sn_est_gpu.py:326), raw normal Re(conj(I) W)/|I|
 * (surface_normal_est.cu:138-144), unit normalisation (image_processor.py:396).
 * normals: float32 [V, 3], NaN outside the mask.  mask (may be NULL): uint8 [V].
 * raw (may be NULL): float32 [V, 3] un-normalised normal, NaN outside the mask.
 * Needs mmn_normals_workspace_bytes() of workspace.
 */
size_t mmn_normals_workspace_bytes(int64_t num_voxels);
int mmn_normals(int64_t num_voxels, const float *image, const float *vote,
                float filter_percent, float *normals, uint8_t *mask, float *raw,
                void *workspace, size_t workspace_bytes, cudaStream_t stream);

/*
 * The two halves of mmn_normals, for a grid split into voxel slabs over several GPUs
 * (the reference splits the voxel range the same way through start_ind,
 * py_image_gpu.py:187,273): the mask threshold needs the maximum |I| over the WHOLE
 * grid, so each slab takes its local maximum, the caller combines them (an all-reduce
 * of one float with MAX), and each slab then finishes its normals against the global
 * value.
 * mmn_image_max_abs: *max_abs (device, one float) = max |image[v]| over the slab.
 * mmn_normals_from_max: as mmn_normals, with max|I| read from *max_abs (device).
 */
int mmn_image_max_abs(int64_t num_voxels, const float *image, float *max_abs,
                      cudaStream_t stream);
int mmn_normals_from_max(int64_t num_voxels, const float *image, const float *vote,
                         const float *max_abs, float filter_percent, float *normals,
                         uint8_t *mask, float *raw, cudaStream_t stream);

/*
 * Connected components (6-connectivity) of a voxel mask, as
 * _find_connected_components does with cc3d.connected_components(mask, connectivity=6)
 * (src/data_processing/sdf.py:94-120).  mask: uint8 [V] (1 = voxel with a valid normal).
 * root: int32 [V], the smallest flat index in the voxel's component (-1 outside the mask);
 * count: int32 [V], the component's voxel count at its root index (0 elsewhere).  The
 * root is a canonical label: it does not depend on the order of the GPU's unions.
 * Needs mmn_components_workspace_bytes() of workspace (the status word).
 */
size_t mmn_components_workspace_bytes(int64_t num_voxels);
int mmn_components(int32_t num_x, int32_t num_y, int32_t num_z, const uint8_t *mask,
                   int32_t *root, int32_t *count, void *workspace, size_t workspace_bytes,
                   cudaStream_t stream);

/*
 * Relative signed distance field of one component by breadth-first integration of the
 * normals (_construct_rsdf_components, src/data_processing/sdf.py:122-224): from voxel
 * `seed` (rsdf 0), every voxel of the component with root `comp_root` receives
 * rsdf[cell] + dot(step * dx, normal[voxel]) from the cell that enqueues it in the
 * reference's FIFO order (neighbours -x, +y, +x, -y, +z, -z), bit for bit.
 * normals: float64 [V, 3] (NaN x-component = no normal); rsdf: float64 [V], written only
 * on the component's voxels (the caller initialises the rest, e.g. to NaN).
 * *visited_count (may be NULL) receives the number of voxels reached.  Synchronises
 * `stream` once per search level (the next level's size decides the launch).
 * Grids up to 357,913,941 voxels.
 */
size_t mmn_rsdf_workspace_bytes(int32_t num_x, int32_t num_y, int32_t num_z);
int mmn_rsdf_component(int32_t num_x, int32_t num_y, int32_t num_z, const double *normals,
                       const int32_t *root, int32_t comp_root, int32_t seed, double dx,
                       double *rsdf, int64_t *visited_count, void *workspace,
                       size_t workspace_bytes, cudaStream_t stream);

/*
 * Channels simulated from isosurfaces of the RSDF (_simulate_channels,
 * src/data_processing/isosurface_optimization.py:116-208, with the ray marching of
 * src/data_processing/cuda/ray_tracing_kernel.cu): for every offset set t and antenna a,
 * width x height rays from the antenna over +-width_fov / +-height_fov degrees march each
 * component's grid (rsdf - taus[t][c]); every hit, refined by one trilinear step, adds
 * exp(j 2 pi d f_k / c) (d the round trip plus range_offset) at every frequency
 * f_k / c = f0_over_c + k * df_over_c, summed over the components.
 * grids: float32 [num_comp][res_x][res_y][res_z], -50 where undefined.  bbox: min x, y, z,
 * max x, y, z (float32, as the marching kernel receives them); voxel_size and lower: the
 * FP32 voxel size and lower corner the refinement step uses.
 */
typedef struct mmn_iso_scene {
    const float *grids;
    int32_t num_comp;
    int32_t res_x, res_y, res_z;
    float bbox[6];
    float voxel_size;
    float lower[3];
    int32_t width, height;
    float width_fov, height_fov;
    double range_offset;
    double f0_over_c, df_over_c;
    int32_t num_wl;
    int32_t reserved;
} mmn_iso_scene;

/* taus: float32 [num_sets][num_comp]; rx_locs: float64 [num_antennas][3]; rx_dirs: float32
 * [num_antennas][3]; channels: complex64 [num_sets][num_antennas][num_wl].  Sets x antennas
 * <= 65535 per call. */
size_t mmn_iso_channels_workspace_bytes(const mmn_iso_scene *scene, int32_t num_sets,
                                        int32_t num_antennas);
int mmn_iso_channels(const mmn_iso_scene *scene, const float *taus, int32_t num_sets,
                     const double *rx_locs, const float *rx_dirs, int32_t num_antennas,
                     float *channels, void *workspace, size_t workspace_bytes,
                     cudaStream_t stream);
/* The rough march of one antenna's rays on component `comp` at offset `tau` (the
 * reference extension's ray_matching outputs): rough hit point, hit voxel index (both -1
 * for no hit) and ray direction, float32 [width * height][3] each. */
int mmn_iso_march(const mmn_iso_scene *scene, int32_t comp, float tau, const double *rx_loc,
                  const float *rx_dir, float *rough, float *voxel, float *direction,
                  cudaStream_t stream);

/*
 * Raw 77 GHz ADC samples (GenericLoader.load_radar_files, src/utils/generic_loader.py:
 * 521-535): raw holds little-endian int16, 8 per sample (I of lanes 0-3, then Q of lanes
 * 0-3); out: complex64 [num_samples][4] (the int16 values are exact in FP32).
 */
int mmn_adc_unpack(const int16_t *raw, int64_t num_samples, float *out, cudaStream_t stream);

/*
 * The antenna position of every radar frame (ImageProcessor.correlate_locs_and_meas,
 * src/data_processing/image_processor.py:74-154): per row (radar file) r and frame j, the
 * trajectory (times ascending [num_points], traj [num_points][dim], 3 <= dim <= 8) is
 * interpolated linearly at created[r] + j * frame_dt as scipy's interp1d does; the frame is
 * kept unless its time is outside the trajectory, it lies within `threshold` of a frame
 * kept earlier in the same row (j > 0; with no frame kept yet in the row, frames j > 0 are
 * dropped, as the reference's minimum over an empty list raises), or the row's file holds
 * fewer than j * frame_stride + samples samples (available[r]; -1 skips the row).
 * optitrack != 0 applies the optitrack axis change (-x, z, y) to kept positions.
 * loc_out: float64 [num_rows][num_frames][optitrack ? 3 : dim]; keep: uint8
 * [num_rows][num_frames]; scratch: int32 [num_rows][num_frames].
 */
int mmn_correlate_poses(const double *times, const double *traj, int64_t num_points,
                        int32_t dim, const double *created, const int64_t *available,
                        int32_t num_rows, int32_t num_frames, double frame_dt, double threshold,
                        int64_t frame_stride, int64_t samples, int32_t optitrack,
                        double *loc_out, uint8_t *keep, int32_t *scratch, cudaStream_t stream);

/*
 * Drop-in for the reference kernel launch `cuda_image`
 * (src/data_processing/cuda/imaging_gpu.cu:12-21, launched at py_image_gpu.py:189-199):
 * same arguments in the same order and meaning (SoA measurements, float scalars,
 * start_ind), plus the launch extent voxel_count (the reference's grid_dim *
 * threads_per_block, py_image_gpu.py:273,187; -1 = to the end of the grid), a
 * workspace and a stream.  Writes p_xyz_r/p_xyz_i for voxels [start_ind,
 * start_ind + voxel_count).  use_interpolated_processing == 0 runs the mixed-precision
 * matched filter; 1 runs the interpolated mode with the reference's arithmetic (bit for
 * bit); 2 runs the interpolated mode's fast form (MMN_MODE_INTERP_FAST).
 */
size_t mmn_cuda_image_workspace_bytes(int num_antennas, int samples_per_meas,
                                      int use_interpolated_processing);
/* Exact workspace for one mmn_cuda_image call (includes the antenna-split partial sums,
 * which depend on the launch extent and the current device). */
size_t mmn_cuda_image_workspace_bytes_for(int num_x, int num_y, int num_z, int num_antennas,
                                          int samples_per_meas, int start_ind, int voxel_count,
                                          int use_interpolated_processing);
int mmn_cuda_image(float *p_xyz_r, float *p_xyz_i, const float *x_locs,
                   const float *y_locs, const float *z_locs, const float *antenna_locs,
                   const float *meas_r, const float *meas_i, const float *rx_offsets,
                   float slope, float wavelength, float fft_spacing, int num_x,
                   int num_y, int num_z, int num_antennas, int num_rx_antennas,
                   int samples_per_meas, int start_ind, int is_ti_radar,
                   int use_interpolated_processing, int voxel_count, void *workspace,
                   size_t workspace_bytes, cudaStream_t stream);

/*
 * Drop-in for the reference kernel launch `cuda_sn_est`
 * (src/data_processing/cuda/surface_normal_est.cu:14-25, launched at
 * py_sn_est_gpu.py:229-246): interpolated-mode normal vote for the listed valid
 * voxels with the reference's arithmetic; writes normals_x/y/z[ind] for
 * ind in [start_ind, min(num_valid_idx, start_ind + count)) (count = -1: all).
 */
size_t mmn_cuda_sn_est_workspace_bytes(int num_antennas, int samples_per_meas);
int mmn_cuda_sn_est(float *normals_x, float *normals_y, float *normals_z,
                    const int *valid_idx_x, const int *valid_idx_y,
                    const int *valid_idx_z, const float *p_xyz_r, const float *p_xyz_i,
                    const float *x_locs, const float *y_locs, const float *z_locs,
                    const float *antenna_locs, const float *meas_r, const float *meas_i,
                    const float *rx_offsets, float slope, float wavelength,
                    float fft_spacing, int num_x, int num_y, int num_z,
                    int num_antennas, int num_rx_antennas, int num_valid_idx,
                    int samples_per_meas, int start_ind, int is_ti_radar, int count,
                    void *workspace, size_t workspace_bytes, cudaStream_t stream);

/*
 * mmn_cuda_sn_est in the fast form of MMN_MODE_INTERP_FAST (no counterpart in the
 * reference): same arguments, valid-voxel list and outputs; the reference's path length
 * and range bin, the phasor from the wrapped FP32 turn count and the hardware
 * sine/cosine, and the weight as one multiply by 1/|I|.
 */
int mmn_cuda_sn_est_fast(float *normals_x, float *normals_y, float *normals_z,
                         const int *valid_idx_x, const int *valid_idx_y,
                         const int *valid_idx_z, const float *p_xyz_r, const float *p_xyz_i,
                         const float *x_locs, const float *y_locs, const float *z_locs,
                         const float *antenna_locs, const float *meas_r, const float *meas_i,
                         const float *rx_offsets, float slope, float wavelength,
                         float fft_spacing, int num_x, int num_y, int num_z,
                         int num_antennas, int num_rx_antennas, int num_valid_idx,
                         int samples_per_meas, int start_ind, int is_ti_radar, int count,
                         void *workspace, size_t workspace_bytes, cudaStream_t stream);

/*
 * FP32 FMA throughput probe (no counterpart in the reference): `blocks` CTAs of 256
 * threads each run 16 independent FFMA chains for `iters` iterations, i.e.
 * blocks*256*iters*32 FLOPs; out: float [blocks*256] sink.  Timed by the caller, it gives
 * the measured FP32 peak that bounds the forward kernels.
 */
int mmn_fp32_peak_probe(int blocks, int iters, float *out, cudaStream_t stream);

/*
 * Bounded-wait check (no counterpart in the reference, whose kernels have no waits): one
 * warp waits on an mbarrier with the same bounded wait the copy pipelines use (which give up
 * after one second), here giving up after `limit_us` microseconds (at most 10 s, else
 * MMN_ERR_INVALID_ARGUMENT).  With `arrive` != 0 the phase is completed first and the wait
 * succeeds; with `arrive` == 0 nothing completes it, the wait runs out and the kernel
 * records MMN_ERR_TIMEOUT in the status word at the start of `workspace` (read and clear it
 * with mmn_read_status) and returns.  Nothing faults and the context stays usable.
 */
int mmn_wait_timeout_probe(uint32_t limit_us, int arrive, void *workspace,
                           cudaStream_t stream);

/*
 * Status word that kernels set when a bounded wait gives up (MMN_ERR_TIMEOUT) -- kept in
 * the first bytes of every workspace.  Synchronises `stream`, copies the word to the
 * host, and clears it.  Returns MMN_OK or the CUDA error; *status receives the word.
 */
int mmn_read_status(void *workspace, int32_t *status, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MMNORM_B200_H */

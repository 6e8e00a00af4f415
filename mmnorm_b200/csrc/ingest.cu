// ingest.cu -- raw ADC frames and the antenna position of every frame, on the GPU.
//
// Reference: GenericLoader.load_radar_files (src/utils/generic_loader.py:521-535, 77 GHz
// .bin files: little-endian int16, 8 per sample = I of lanes 0-3 then Q of lanes 0-3) and
// ImageProcessor.correlate_locs_and_meas (src/data_processing/image_processor.py:74-154):
// the robot trajectory is interpolated linearly (scipy interp1d, :37-62) at the start time
// of every frame j of every radar file (created_ts + j * (sweep_time + periodicity)); a
// frame is dropped when its time lies outside the trajectory, when it is within
// 3/16 wavelength of a frame already kept from the same file, or when the file holds too
// few samples for it; otherwise its position and samples are kept.
//
// One warp per radar file: the frames of a file depend on each other (the distance test
// looks at the frames kept before), so a file's frames run in order, and the lanes split
// the distance test over the kept frames.  The interpolation repeats numpy.interp (which
// scipy's linear interp1d uses for float64 columns): slope * (x - t_j) + y_j with one
// rounding per operation, so positions and decisions are numpy's.
#include "mmn_internal.cuh"

namespace mmn {
namespace {

__global__ void adc_unpack_kernel(const int16_t *__restrict__ raw, int64_t samples,
                                  float2 *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // (sample, lane)
    if (i >= samples * 4) return;
    const int64_t s = i >> 2;
    const int l = (int)(i & 3);
    out[i] = make_float2((float)raw[8 * s + l], (float)raw[8 * s + 4 + l]);
}

struct PoseArgs {
    const double *times;     // [n] ascending
    const double *traj;      // [n][dim]
    int64_t n;
    int dim;
    const double *created;   // [rows]
    const int64_t *avail;    // [rows] samples in the row's file (-1: no file / skipped row)
    int rows, frames;
    double frame_dt;         // sweep_time + periodicity
    double threshold;        // 3/16 wavelength
    int64_t frame_stride;    // samples_per_chirp * num_chirps
    int64_t samples;         // samples_per_chirp
    int optitrack;           // apply the optitrack frame change before keeping
    double *loc_out;         // [rows][frames][dim_out]
    uint8_t *keep;           // [rows][frames]
    int32_t *kept;           // [rows][frames] scratch: indices of kept frames
};

__global__ void pose_kernel(const PoseArgs a) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= a.rows) return;
    const int dim_out = a.optitrack ? 3 : a.dim;
    uint8_t *keep = a.keep + (int64_t)row * a.frames;
    double *locs = a.loc_out + (int64_t)row * a.frames * dim_out;
    int32_t *kept = a.kept + (int64_t)row * a.frames;
    for (int j = lane; j < a.frames; j += 32) keep[j] = 0;
    __syncwarp();
    if (a.avail[row] < 0) return;
    int nk = 0;
    const double x0 = a.times[0], xn = a.times[a.n - 1];
    for (int j = 0; j < a.frames; ++j) {
        const double x = __dadd_rn(a.created[row], __dmul_rn((double)j, a.frame_dt));
        if (x < x0 || x > xn) continue;  // interp1d raises: the frame is skipped
        // numpy.interp (scipy's interp1d hands float64 columns to it): j with
        // t[j] <= x < t[j+1]; exact knots return their value; else
        // slope * (x - t[j]) + y[j], slope = (y[j+1] - y[j]) / (t[j+1] - t[j])
        int64_t lo = 0, hi = a.n;  // first index with t > x
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (a.times[mid] <= x) lo = mid + 1; else hi = mid;
        }
        const int64_t k = lo - 1;
        double loc[8];
        for (int d = 0; d < a.dim && d < 8; ++d) {
            if (k >= a.n - 1 || a.times[k] == x) {
                loc[d] = a.traj[k * a.dim + d];
            } else {
                const double y0 = a.traj[k * a.dim + d], y1 = a.traj[(k + 1) * a.dim + d];
                const double slope = __ddiv_rn(__dsub_rn(y1, y0),
                                               __dsub_rn(a.times[k + 1], a.times[k]));
                loc[d] = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, a.times[k])), y0);
            }
        }
        if (j != 0) {
            if (nk == 0) continue;  // the minimum over no kept frames raises: skipped
            bool close = false;
            for (int i = lane; i < nk; i += 32) {
                const double *q = locs + (int64_t)kept[i] * dim_out;
                const double ex = __dsub_rn(q[0], loc[0]), ey = __dsub_rn(q[1], loc[1]),
                             ez = __dsub_rn(q[2], loc[2]);
                const double s = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)),
                                           __dmul_rn(ez, ez));
                if (__dsqrt_rn(s) < a.threshold) close = true;
            }
            if (__any_sync(0xffffffffu, close)) continue;
        }
        if ((int64_t)j * a.frame_stride + a.samples > a.avail[row]) continue;  // short file
        if (lane == 0) {
            double *dst = locs + (int64_t)j * dim_out;
            if (a.optitrack) {
                dst[0] = -loc[0];
                dst[1] = loc[2];
                dst[2] = loc[1];
            } else {
                for (int d = 0; d < a.dim && d < 8; ++d) dst[d] = loc[d];
            }
            keep[j] = 1;
            kept[nk] = j;
        }
        ++nk;
        __syncwarp();
    }
}

}  // namespace
}  // namespace mmn

extern "C" int mmn_adc_unpack(const int16_t *raw, int64_t num_samples, float *out,
                              cudaStream_t stream) {
    if (num_samples < 0) return MMN_ERR_INVALID_ARGUMENT;
    if (num_samples == 0) return MMN_OK;
    if (!raw || !out) return MMN_ERR_NULL_POINTER;
    const int64_t n = num_samples * 4;
    mmn::adc_unpack_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
        raw, num_samples, reinterpret_cast<float2 *>(out));
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

extern "C" int mmn_correlate_poses(const double *times, const double *traj, int64_t num_points,
                                   int32_t dim, const double *created, const int64_t *available,
                                   int32_t num_rows, int32_t num_frames, double frame_dt,
                                   double threshold, int64_t frame_stride, int64_t samples,
                                   int32_t optitrack, double *loc_out, uint8_t *keep,
                                   int32_t *scratch, cudaStream_t stream) {
    if (num_points < 2 || dim < 3 || dim > 8 || num_rows < 0 || num_frames < 0 ||
        frame_stride < 1 || samples < 1)
        return MMN_ERR_INVALID_ARGUMENT;
    if (num_rows == 0 || num_frames == 0) return MMN_OK;
    if (!times || !traj || !created || !available || !loc_out || !keep || !scratch)
        return MMN_ERR_NULL_POINTER;
    mmn::PoseArgs a;
    a.times = times;
    a.traj = traj;
    a.n = num_points;
    a.dim = dim;
    a.created = created;
    a.avail = available;
    a.rows = num_rows;
    a.frames = num_frames;
    a.frame_dt = frame_dt;
    a.threshold = threshold;
    a.frame_stride = frame_stride;
    a.samples = samples;
    a.optitrack = optitrack;
    a.loc_out = loc_out;
    a.keep = keep;
    a.kept = scratch;
    const int warps = 4;
    mmn::pose_kernel<<<(num_rows + warps - 1) / warps, warps * 32, 0, stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

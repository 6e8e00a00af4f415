// isosurface.cu -- mmWave channels simulated from an isosurface of the RSDF: ray marching
// fused with the channel synthesis.
//
// Reference: _simulate_channels (src/data_processing/isosurface_optimization.py:116-208)
// and the ray-marching extension it calls (src/data_processing/cuda/ray_tracing_kernel.cu:
// GenerateRay :60-120, ValueAt :200-290, Intersect :292-400).  For one antenna and one
// isosurface offset tau per RSDF component, width x height rays leave the antenna over the
// field of view; each marches the grid (rsdf - tau) with steps equal to the trilinear SDF
// value (MIN_STEP where a corner is undefined) until the value drops below one voxel; the
// hit is refined by one more step of the trilinear value at the hit voxel
// (_compute_intersection_pos :66-92), and every hit adds exp(j 2 pi d / lambda_k), d the
// round trip (+0.15 m for the TI radar), to the antenna's channel at every wavelength.
//
// Ray generation and marching repeat the reference kernel's FP32 arithmetic expression for
// expression (including its float-valued flat index), so the hits and rough positions are
// the reference's; the refinement repeats the torch expressions with one rounding per
// operation, as torch evaluates them; the distance is FP64 (the reference subtracts the
// FP32 hit from the FP64 antenna position).  The synthesis evaluates
// exp(j 2 pi d f_k / c) from an exact fixed-point phase per (hit, wavelength) and the
// hardware sincos on the wrapped angle (f_k uniform, f_k = c / lambda_k).
//
// Work item = (offset set t, antenna a); grid = (ray blocks, items).  A block takes every
// blocks-per-item-th tile of 256 rays, marches them through every component, collects the
// hits in ray order and adds them to its partial channel [K]; a second kernel adds the
// blocks' partials in block order (FP64) -- deterministic run to run.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "mmn_internal.cuh"

namespace mmn {
namespace {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kUndef = -50.f;
constexpr float kMinStep = 0.005;   // a double literal narrowed to float, as the reference
constexpr int kMaxSteps = 1000;
constexpr int kIsoThreads = 256;

struct IsoParams {
    const float *grids;        // [C][NX][NY][NZ] RSDF, kUndef where undefined
    const float *taus;         // [T][C] offsets (already clipped to their bounds)
    const double *rx_locs;     // [A][3] antenna positions (FP64, for the distance)
    const float *rx_dirs;      // [A][3]
    int num_comp, num_ant, num_items;
    int width, height;
    float width_fov, height_fov;
    float bb_min_x, bb_min_y, bb_min_z, bb_max_x, bb_max_y, bb_max_z;
    int res_x, res_y, res_z;
    float voxel_size_ref;      // the voxel size the refinement step uses (voxel_size)
    float lower_x, lower_y, lower_z;  // bounding_box_lower (FP32)
    double range_offset;       // 0.15 for the TI radar, else 0
    double f0_over_c, df_over_c;  // f_k / c = f0_over_c + k * df_over_c (1/m)
    int num_wl;
    float2 *partial;           // [items][blocks][K]
    int32_t *block_hits;       // [items][blocks]
    int blocks_per_item;
    int32_t *status;
};

__device__ __forceinline__ float deg_to_rad(const float &deg) { return (deg * (kPiF / 180.f)); }

__device__ __forceinline__ float vlen(const float x, const float y, const float z) {
    return sqrtf(powf(x, 2) + powf(y, 2) + powf(z, 2));
}

// the antenna's view frame (w along the antenna direction, u = up x w, v = w x u) and the
// field of view in radians: the same for every ray of an antenna, formed once per block
struct RayBasis {
    float w_x, w_y, w_z, u_x, u_y, u_z, v_x, v_y, v_z, horiz_fov, vert_fov;
};

__device__ RayBasis ray_basis(const IsoParams &p, float rdx, float rdy, float rdz) {
    RayBasis b;
    const float up_x = 1, up_y = 0, up_z = 0;
    b.vert_fov = deg_to_rad(p.height_fov);
    b.horiz_fov = deg_to_rad(p.width_fov);
    b.w_x = (rdx) / vlen(rdx, rdy, rdz);
    b.w_y = (rdy) / vlen(rdx, rdy, rdz);
    b.w_z = (rdz) / vlen(rdx, rdy, rdz);
    const float cuw_x = up_y * b.w_z - up_z * b.w_y;
    const float cuw_y = up_z * b.w_x - up_x * b.w_z;
    const float cuw_z = up_x * b.w_y - up_y * b.w_x;
    b.u_x = (cuw_x) / vlen(cuw_x, cuw_y, cuw_z);
    b.u_y = (cuw_y) / vlen(cuw_x, cuw_y, cuw_z);
    b.u_z = (cuw_z) / vlen(cuw_x, cuw_y, cuw_z);
    b.v_x = b.w_y * b.u_z - b.w_z * b.u_y;
    b.v_y = b.w_z * b.u_x - b.w_x * b.u_z;
    b.v_z = b.w_x * b.u_y - b.w_y * b.u_x;
    return b;
}

// ray direction of pixel (px, py)
__device__ void ray_direction(const IsoParams &p, const RayBasis &b, int px, int py, float &dx,
                              float &dy, float &dz) {
    const float horiz_fov = b.horiz_fov, vert_fov = b.vert_fov;
    // the angle is formed in double (a float plus 0.5) and narrowed, as the reference does
    const float horiz_angle = -horiz_fov + (horiz_fov*2) * (__int2float_rd(px) + 0.5)/ __int2float_rd(p.width);
    const float vert_angle = -vert_fov + (vert_fov*2) * (__int2float_rd(py) + 0.5)/ __int2float_rd(p.height);
    const float view_plane_x = tan(horiz_angle);
    const float view_plane_y = tan(vert_angle);
    const float s_x = view_plane_x * b.u_x + view_plane_y * b.v_x - b.w_x;
    const float s_y = view_plane_x * b.u_y + view_plane_y * b.v_y - b.w_y;
    const float s_z = view_plane_x * b.u_z + view_plane_y * b.v_z - b.w_z;
    const float len = vlen(s_x, s_y, s_z);
    dx = s_x / len;
    dy = s_y / len;
    dz = s_z / len;
}

__device__ __forceinline__ bool inside_box(const IsoParams &p, float x, float y, float z) {
    return (x >= p.bb_min_x) && (x <= p.bb_max_x) && (y >= p.bb_min_y) && (y <= p.bb_max_y) &&
           (z >= p.bb_min_z) && (z <= p.bb_max_z);
}

// distance along the ray to the bounding box from outside (-1: none)
__device__ float box_distance(const IsoParams &p, float px, float py, float pz, float dx, float dy,
                              float dz) {
    float dist = -1.f;
    dx = dx / vlen(dx, dy, dz);
    dy = dy / vlen(dx, dy, dz);
    dz = dz / vlen(dx, dy, dz);
    const float vs[3] = {px, py, pz};
    const float ds[3] = {dx, dy, dz};
    const float lo[3] = {p.bb_min_x, p.bb_min_y, p.bb_min_z};
    const float hi[3] = {p.bb_max_x, p.bb_max_y, p.bb_max_z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v = vs[k], d = ds[k];
        if (dist == -1) {
            if ((v < lo[k]) && (d > 0)) { dist = (lo[k] - v) / d; }
            if ((v > hi[k]) && (d < 0)) { dist = (hi[k] - v) / d; }
        } else {
            if ((v < lo[k]) && (d > 0)) { dist = fmaxf(dist, (lo[k] - v) / d); }
            if ((v > hi[k]) && (d < 0)) { dist = fmaxf(dist, (hi[k] - v) / d); }
        }
    }
    return dist;
}

// the reference's flat index: integer parts recombined in FP32 (exact below 2^24 voxels)
__device__ __forceinline__ int flat_index(float const x, float const y, float const z, int const rx,
                                          int const ry, int const rz) {
    (void)rx;
    return __int2float_rd(z) + __int2float_rd(y) * rz + __int2float_rd(x) * rz * ry;
}

__device__ __forceinline__ float grid_at(const float *g, float tau, int idx, int n, bool &ok) {
    if (idx < 0 || idx >= n) {
        ok = false;
        return 0.f;
    }
    return __fsub_rn(g[idx], tau);
}

// signed distance at a point (the reference's ValueAt); ok=false if an index left the grid
__device__ float value_at(const IsoParams &p, const float *g, float tau, float px, float py, float pz,
                          float dx, float dy, float dz, bool first_time, bool &ok) {
    if (!inside_box(p, px, py, pz)) {
        if (first_time)
            return box_distance(p, px, py, pz, dx, dy, dz) + 0.00001f;
        return -1;
    }
    const int n = p.res_x * p.res_y * p.res_z;
    const float voxel_size = (p.bb_max_y - p.bb_min_y) / (p.res_y - 1);
    float mx = floorf((px - p.bb_min_x) / voxel_size);
    float my = floorf((py - p.bb_min_y) / voxel_size);
    float mz = floorf((pz - p.bb_min_z) / voxel_size);
    if (mx == (p.bb_max_x - p.bb_min_x) / voxel_size) mx = (p.bb_max_x - p.bb_min_x) / voxel_size - 1;
    if (my == (p.bb_max_y - p.bb_min_y) / voxel_size) my = (p.bb_max_y - p.bb_min_y) / voxel_size - 1;
    if (mz == (p.bb_max_z - p.bb_min_z) / voxel_size) mz = (p.bb_max_z - p.bb_min_z) / voxel_size - 1;
    const int rx = p.res_x, ry = p.res_y, rz = p.res_z;
    const float g000 = grid_at(g, tau, flat_index(mx, my, mz, rx, ry, rz), n, ok);
    const float g010 = grid_at(g, tau, flat_index(mx, my + 1, mz, rx, ry, rz), n, ok);
    const float g001 = grid_at(g, tau, flat_index(mx, my, mz + 1, rx, ry, rz), n, ok);
    const float g011 = grid_at(g, tau, flat_index(mx, my + 1, mz + 1, rx, ry, rz), n, ok);
    const float g100 = grid_at(g, tau, flat_index(mx + 1, my, mz, rx, ry, rz), n, ok);
    const float g110 = grid_at(g, tau, flat_index(mx + 1, my + 1, mz, rx, ry, rz), n, ok);
    const float g101 = grid_at(g, tau, flat_index(mx + 1, my, mz + 1, rx, ry, rz), n, ok);
    const float g111 = grid_at(g, tau, flat_index(mx + 1, my + 1, mz + 1, rx, ry, rz), n, ok);
    if (g000 < kUndef + 10 || g010 < kUndef + 10 || g001 < kUndef + 10 || g011 < kUndef + 10 ||
        g100 < kUndef + 10 || g110 < kUndef + 10 || g101 < kUndef + 10 || g111 < kUndef + 10)
        return kMinStep;
    const float tx = (px - (p.bb_min_x + mx * voxel_size)) / voxel_size;
    const float ex_y0z0 = (1.f - tx) * g000 + tx * g100;
    const float ex_y1z0 = (1.f - tx) * g010 + tx * g110;
    const float ex_y0z1 = (1.f - tx) * g001 + tx * g101;
    const float ex_y1z1 = (1.f - tx) * g011 + tx * g111;
    const float ty = (py - (p.bb_min_y + my * voxel_size)) / voxel_size;
    const float fz0 = (1.f - ty) * ex_y0z0 + ty * ex_y1z0;
    const float fz1 = (1.f - ty) * ex_y0z1 + ty * ex_y1z1;
    const float tz = (pz - (p.bb_min_z + mz * voxel_size)) / voxel_size;
    return (1.f - tz) * fz0 + tz * fz1;
}

// marches one ray; on a hit returns true with the rough point and its voxel index
__device__ bool march(const IsoParams &p, const float *g, float tau, float ox, float oy, float oz,
                      float dx, float dy, float dz, float &hx, float &hy, float &hz, float &vx,
                      float &vy, float &vz) {
    const float voxel_size = (p.bb_max_y - p.bb_min_y) / (p.res_y - 1);
    bool first_time = true;
    float depth = 0;
    for (int steps = 0; steps < kMaxSteps; steps++) {
        const float rx = ox + depth * dx;
        const float ry = oy + depth * dy;
        const float rz = oz + depth * dz;
        bool ok = true;
        const float distance = value_at(p, g, tau, rx, ry, rz, dx, dy, dz, first_time, ok);
        if (!ok) return false;
        first_time = false;
        if (distance == -1) return false;
        if (distance < voxel_size && distance) {
            vx = floorf((rx - p.bb_min_x) / voxel_size);
            vy = floorf((ry - p.bb_min_y) / voxel_size);
            vz = floorf((rz - p.bb_min_z) / voxel_size);
            if (vx == p.res_x - 1) vx = vx - 1;
            if (vy == p.res_y - 1) vy = vy - 1;
            if (vz == p.res_z - 1) vz = vz - 1;
            hx = rx;
            hy = ry;
            hz = rz;
            return true;
        }
        depth += distance;
    }
    return false;
}

// _compute_intersection_pos for one hit, one rounding per torch operation; ok=false when the
// hit's voxel is not inside the grid (the reference would index outside its tensor)
__device__ bool refine(const IsoParams &p, const float *g, float tau, float hx, float hy, float hz,
                       float vx, float vy, float vz, float dx, float dy, float dz, float &ix,
                       float &iy, float &iz) {
    const int x = (int)(vx == -1.f ? 0.f : vx), y = (int)(vy == -1.f ? 0.f : vy),
              z = (int)(vz == -1.f ? 0.f : vz);
    if (x < 0 || y < 0 || z < 0 || x + 1 >= p.res_x || y + 1 >= p.res_y || z + 1 >= p.res_z)
        return false;
    auto at = [&](int a, int b, int c) {
        return __fsub_rn(g[((int64_t)a * p.res_y + b) * p.res_z + c], tau);
    };
    const float vs = p.voxel_size_ref;
    const float mnx = __fadd_rn(p.lower_x, __fmul_rn(vx, vs));
    const float mny = __fadd_rn(p.lower_y, __fmul_rn(vy, vs));
    const float mnz = __fadd_rn(p.lower_z, __fmul_rn(vz, vs));
    auto lerp = [](float t, float a, float b) {
        return __fadd_rn(__fmul_rn(__fsub_rn(1.f, t), a), __fmul_rn(t, b));
    };
    const float tx = __fdiv_rn(__fsub_rn(hx, mnx), vs);
    const float ex_y0z0 = lerp(tx, at(x, y, z), at(x + 1, y, z));
    const float ex_y1z0 = lerp(tx, at(x, y + 1, z), at(x + 1, y + 1, z));
    const float ex_y0z1 = lerp(tx, at(x, y, z + 1), at(x + 1, y, z + 1));
    const float ex_y1z1 = lerp(tx, at(x, y + 1, z + 1), at(x + 1, y + 1, z + 1));
    const float ty = __fdiv_rn(__fsub_rn(hy, mny), vs);
    const float fz0 = lerp(ty, ex_y0z0, ex_y1z0);
    const float fz1 = lerp(ty, ex_y0z1, ex_y1z1);
    const float tz = __fdiv_rn(__fsub_rn(hz, mnz), vs);
    const float sdf = lerp(tz, fz0, fz1);
    ix = __fadd_rn(hx, __fmul_rn(dx, sdf));
    iy = __fadd_rn(hy, __fmul_rn(dy, sdf));
    iz = __fadd_rn(hz, __fmul_rn(dz, sdf));
    return true;
}

__global__ void __launch_bounds__(kIsoThreads) iso_channel_kernel(const IsoParams p) {
    __shared__ unsigned long long s_ph0[kIsoThreads], s_stp[kIsoThreads];
    __shared__ int s_warp[kIsoThreads / 32 + 1];
    const int item = blockIdx.y;
    const int t = item / p.num_ant, a = item % p.num_ant;
    const int npix = p.width * p.height;
    const int ntiles = (npix + kIsoThreads - 1) / kIsoThreads;
    const float eye_x = (float)p.rx_locs[3 * a], eye_y = (float)p.rx_locs[3 * a + 1],
                eye_z = (float)p.rx_locs[3 * a + 2];
    const RayBasis basis = ray_basis(p, p.rx_dirs[3 * a], p.rx_dirs[3 * a + 1], p.rx_dirs[3 * a + 2]);
    const int64_t ncell = (int64_t)p.res_x * p.res_y * p.res_z;
    const int64_t bslot = (int64_t)item * p.blocks_per_item + blockIdx.x;
    float2 *dst = p.partial + bslot * p.num_wl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int total = 0;  // block-uniform: hits added to dst so far
    // this block's tiles of 256 rays, in order; every component's isosurface in turn (the
    // reference sums the components' channels)
    for (int tile = blockIdx.x; tile < ntiles; tile += p.blocks_per_item) {
        const int pixel = tile * kIsoThreads + threadIdx.x;
        float dx = 0.f, dy = 0.f, dz = 0.f;
        if (pixel < npix) ray_direction(p, basis, pixel % p.width, pixel / p.width, dx, dy, dz);
        for (int c = 0; c < p.num_comp; ++c) {
            const float *g = p.grids + (int64_t)c * ncell;
            const float tau = p.taus[(int64_t)t * p.num_comp + c];
            bool hit = false;
            double d = 0.0;
            if (pixel < npix) {
                float hx, hy, hz, vx, vy, vz, ix, iy, iz;
                if (march(p, g, tau, eye_x, eye_y, eye_z, dx, dy, dz, hx, hy, hz, vx, vy, vz) &&
                    refine(p, g, tau, hx, hy, hz, vx, vy, vz, dx, dy, dz, ix, iy, iz)) {
                    const double ex = p.rx_locs[3 * a] - (double)ix;
                    const double ey = p.rx_locs[3 * a + 1] - (double)iy;
                    const double ez = p.rx_locs[3 * a + 2] - (double)iz;
                    d = sqrt(ex * ex + ey * ey + ez * ez) * 2.0 + p.range_offset;
                    hit = true;
                }
            }
            // the hits of this tile and component, compacted in ray order
            const unsigned ball = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) s_warp[warp] = __popc(ball);
            __syncthreads();
            if (threadIdx.x == 0) {
                int run = 0;
                for (int w = 0; w < kIsoThreads / 32; ++w) {
                    const int cnt = s_warp[w];
                    s_warp[w] = run;
                    run += cnt;
                }
                s_warp[kIsoThreads / 32] = run;
            }
            __syncthreads();
            if (hit) {
                const int slot = s_warp[warp] + __popc(ball & ((1u << lane) - 1u));
                s_ph0[slot] = turns_to_fixed(d * p.f0_over_c);
                s_stp[slot] = turns_to_fixed(d * p.df_over_c);
            }
            __syncthreads();
            const int nh = s_warp[kIsoThreads / 32];
            if (nh > 0) {
                for (int k = threadIdx.x; k < p.num_wl; k += kIsoThreads) {
                    float sr = 0.f, si = 0.f;
                    for (int h = 0; h < nh; ++h) {
                        float cs, sn;
                        fixed_cis(s_ph0[h] + (unsigned long long)k * s_stp[h], cs, sn);
                        sr += cs;
                        si += sn;
                    }
                    if (total > 0) {
                        const float2 o = dst[k];
                        sr += o.x;
                        si += o.y;
                    }
                    dst[k] = make_float2(sr, si);
                }
            }
            total += nh;
            __syncthreads();  // the shared hit lists are refilled by the next pass
        }
    }
    if (threadIdx.x == 0) p.block_hits[bslot] = total;
}

// channel[item][k] = sum over the item's blocks (in block order) of their partials
__global__ void iso_reduce_kernel(const IsoParams p, float2 *__restrict__ channel) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)p.num_items * p.num_wl) return;
    const int item = (int)(idx / p.num_wl), k = (int)(idx % p.num_wl);
    double sr = 0.0, si = 0.0;
    for (int b = 0; b < p.blocks_per_item; ++b) {
        const int64_t bslot = (int64_t)item * p.blocks_per_item + b;
        if (p.block_hits[bslot] == 0) continue;
        const float2 v = p.partial[bslot * p.num_wl + k];
        sr += v.x;
        si += v.y;
    }
    channel[idx] = make_float2((float)sr, (float)si);
}

// rough hits of one antenna's rays (for tests against the reference extension): per pixel
// the rough point (-1 if none), the voxel index (-1 if none) and the ray direction
__global__ void iso_march_debug_kernel(const IsoParams p, int comp, float tau, int ant,
                                       float *rough, float *voxel, float *dir) {
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= p.width * p.height) return;
    float dx, dy, dz;
    const RayBasis basis =
        ray_basis(p, p.rx_dirs[3 * ant], p.rx_dirs[3 * ant + 1], p.rx_dirs[3 * ant + 2]);
    ray_direction(p, basis, pixel % p.width, pixel / p.width, dx, dy, dz);
    const int64_t ncell = (int64_t)p.res_x * p.res_y * p.res_z;
    float hx = -1, hy = -1, hz = -1, vx = -1, vy = -1, vz = -1;
    if (!march(p, p.grids + comp * ncell, tau, (float)p.rx_locs[3 * ant],
               (float)p.rx_locs[3 * ant + 1], (float)p.rx_locs[3 * ant + 2], dx, dy, dz, hx, hy,
               hz, vx, vy, vz)) {
        hx = hy = hz = vx = vy = vz = -1;
    }
    rough[3 * pixel] = hx;
    rough[3 * pixel + 1] = hy;
    rough[3 * pixel + 2] = hz;
    voxel[3 * pixel] = vx;
    voxel[3 * pixel + 1] = vy;
    voxel[3 * pixel + 2] = vz;
    dir[3 * pixel] = dx;
    dir[3 * pixel + 1] = dy;
    dir[3 * pixel + 2] = dz;
}

}  // namespace
}  // namespace mmn

// ----------------------------------------------------------------------------- C ABI
// (the ABI types come in through mmn_internal.cuh)

namespace {
constexpr size_t kIsoStatus = 256;
inline size_t iso_up(size_t x) { return (x + 255) & ~(size_t)255; }

int iso_check(const mmn_iso_scene *s) {
    if (!s) return MMN_ERR_NULL_POINTER;
    if (!s->grids) return MMN_ERR_NULL_POINTER;
    if (s->num_comp < 1 || s->res_x < 2 || s->res_y < 2 || s->res_z < 2 || s->width < 1 ||
        s->height < 1 || s->num_wl < 1)
        return MMN_ERR_INVALID_ARGUMENT;
    if ((int64_t)s->res_x * s->res_y * s->res_z >= ((int64_t)1 << 31)) return MMN_ERR_TOO_LARGE;
    if ((int64_t)s->width * s->height >= ((int64_t)1 << 31)) return MMN_ERR_TOO_LARGE;
    return MMN_OK;
}

// ray-tile blocks per work item: at most 8 per SM (each loops over its share of the tiles)
int64_t iso_blocks(const mmn_iso_scene *s) {
    const int64_t npix = (int64_t)s->width * s->height;
    const int64_t tiles = (npix + mmn::kIsoThreads - 1) / mmn::kIsoThreads;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::min<int64_t>(tiles, (int64_t)sms * 8);
}

mmn::IsoParams iso_params(const mmn_iso_scene *s) {
    mmn::IsoParams p;
    std::memset(&p, 0, sizeof(p));
    p.grids = s->grids;
    p.num_comp = s->num_comp;
    p.width = s->width;
    p.height = s->height;
    p.width_fov = s->width_fov;
    p.height_fov = s->height_fov;
    p.bb_min_x = s->bbox[0];
    p.bb_min_y = s->bbox[1];
    p.bb_min_z = s->bbox[2];
    p.bb_max_x = s->bbox[3];
    p.bb_max_y = s->bbox[4];
    p.bb_max_z = s->bbox[5];
    p.res_x = s->res_x;
    p.res_y = s->res_y;
    p.res_z = s->res_z;
    p.voxel_size_ref = s->voxel_size;
    p.lower_x = s->lower[0];
    p.lower_y = s->lower[1];
    p.lower_z = s->lower[2];
    p.range_offset = s->range_offset;
    p.f0_over_c = s->f0_over_c;
    p.df_over_c = s->df_over_c;
    p.num_wl = s->num_wl;
    return p;
}
}  // namespace

extern "C" size_t mmn_iso_channels_workspace_bytes(const mmn_iso_scene *s, int32_t num_sets,
                                                   int32_t num_antennas) {
    if (iso_check(s) != MMN_OK || num_sets < 1 || num_antennas < 1) return 0;
    const int64_t blocks = iso_blocks(s);
    const int64_t items = (int64_t)num_sets * num_antennas;
    return kIsoStatus + iso_up((size_t)items * blocks * sizeof(int32_t)) +
           iso_up((size_t)items * blocks * s->num_wl * sizeof(float2));
}

extern "C" int mmn_iso_channels(const mmn_iso_scene *s, const float *taus, int32_t num_sets,
                                const double *rx_locs, const float *rx_dirs,
                                int32_t num_antennas, float *channels, void *workspace,
                                size_t workspace_bytes, cudaStream_t stream) {
    int rc = iso_check(s);
    if (rc != MMN_OK) return rc;
    if (!taus || !rx_locs || !rx_dirs || !channels) return MMN_ERR_NULL_POINTER;
    if (num_sets < 1 || num_antennas < 1) return MMN_ERR_INVALID_ARGUMENT;
    const int64_t items = (int64_t)num_sets * num_antennas;
    if (items > 65535) return MMN_ERR_TOO_LARGE;  // grid.y
    const size_t need = mmn_iso_channels_workspace_bytes(s, num_sets, num_antennas);
    if (!workspace || workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255))
        return MMN_ERR_WORKSPACE;
    const int blocks = (int)iso_blocks(s);
    unsigned char *w = static_cast<unsigned char *>(workspace);
    mmn::IsoParams p = iso_params(s);
    p.taus = taus;
    p.rx_locs = rx_locs;
    p.rx_dirs = rx_dirs;
    p.num_ant = num_antennas;
    p.num_items = (int)items;
    p.blocks_per_item = blocks;
    p.status = reinterpret_cast<int32_t *>(w);
    p.block_hits = reinterpret_cast<int32_t *>(w + kIsoStatus);
    p.partial = reinterpret_cast<float2 *>(w + kIsoStatus +
                                           iso_up((size_t)items * blocks * sizeof(int32_t)));
    if (cudaMemsetAsync(w, 0, kIsoStatus, stream) != cudaSuccess) return MMN_ERR_CUDA;
    mmn::iso_channel_kernel<<<dim3(blocks, (unsigned)items), mmn::kIsoThreads, 0, stream>>>(p);
    const int64_t n = items * s->num_wl;
    mmn::iso_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
        p, reinterpret_cast<float2 *>(channels));
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

extern "C" int mmn_iso_march(const mmn_iso_scene *s, int32_t comp, float tau,
                             const double *rx_loc, const float *rx_dir, float *rough,
                             float *voxel, float *direction, cudaStream_t stream) {
    int rc = iso_check(s);
    if (rc != MMN_OK) return rc;
    if (!rx_loc || !rx_dir || !rough || !voxel || !direction) return MMN_ERR_NULL_POINTER;
    if (comp < 0 || comp >= s->num_comp) return MMN_ERR_INVALID_ARGUMENT;
    mmn::IsoParams p = iso_params(s);
    p.rx_locs = rx_loc;
    p.rx_dirs = rx_dir;
    p.num_ant = 1;
    const int64_t npix = (int64_t)s->width * s->height;
    mmn::iso_march_debug_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, stream>>>(
        p, comp, tau, 0, rough, voxel, direction);
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

// rsdf.cu -- connected components of the normal mask and the relative signed distance
// field (RSDF) integrated from the normals by breadth-first search, on the GPU.
//
// Reference: src/data_processing/sdf.py:94-120 (_find_connected_components, which calls
// cc3d.connected_components(mask, connectivity=6)) and sdf.py:122-224
// (_construct_rsdf_components): for each valid component a FIFO breadth-first search
// from a seed voxel visits the 6-neighbours in the order (-x, +y, +x, -y, +z, -z) and sets
//     rsdf[adj] = rsdf[cell] + dot(step * dx, normal[adj])            (sdf.py:222)
// when it enqueues adj.  The value a voxel receives depends on which cell enqueued it,
// i.e. on the queue order, so the search here is level-synchronous but keeps that order
// exactly:
//   * the frontier of level k is stored in queue order;
//   * every (frontier position i, direction d) that reaches an unvisited voxel of the
//     component bids key 6*i + d for it (64-bit atomicMin): the smallest key is the cell
//     that dequeues first, which is the cell that enqueues the voxel sequentially;
//   * the winning bids, read in key order (an exclusive scan over the 6*|frontier| slots),
//     are the next level's queue order -- the order in which the sequential search appends
//     them.
// The increment is computed as numpy's dot of two 3-vectors: a running FP64 sum of the
// three products, without contraction, so the values are the reference's bit for bit.
//
// Components: lock-free union-find over the +x/+y/+z neighbours, always linking the larger
// root under the smaller, so every component ends with the smallest flat index in it as its
// root, whatever the order of the unions.  Every retry loop is bounded; a bound that runs
// out records MMN_ERR_TIMEOUT in the status word.
#include <cstring>

#include "mmn_internal.cuh"

namespace mmn {
namespace {

// parent[x] <= x always (atomicMin only lowers it), so paths strictly decrease and every
// loop below ends by construction; the bounds only guard against a broken invariant
constexpr int kUfMaxSteps = 1 << 26;   // steps of one find
constexpr int kUfMaxRetries = 1 << 16; // link attempts of one union

// parent entries change under other threads' atomicMin: read them through volatile so every
// step loads the current value
__device__ __forceinline__ int32_t uf_find(const int32_t *parent, int32_t a, int32_t *status) {
    const volatile int32_t *vp = parent;
    for (int s = 0; s < kUfMaxSteps; ++s) {
        const int32_t p = vp[a];
        if (p == a) return a;
        a = p;
    }
    set_status(status, MMN_ERR_TIMEOUT);
    return a;
}

__device__ void uf_union(int32_t *parent, int32_t a, int32_t b, int32_t *status) {
    for (int s = 0; s < kUfMaxRetries; ++s) {
        a = uf_find(parent, a, status);
        b = uf_find(parent, b, status);
        if (a == b) return;
        if (a < b) {
            const int32_t old = atomicMin(&parent[b], a);
            if (old == b) return;
            b = old;
        } else {
            const int32_t old = atomicMin(&parent[a], b);
            if (old == a) return;
            a = old;
        }
    }
    set_status(status, MMN_ERR_TIMEOUT);
}

__global__ void cc_init_kernel(const uint8_t *__restrict__ mask, int64_t n,
                               int32_t *__restrict__ parent, int32_t *__restrict__ count) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    parent[v] = mask[v] ? (int32_t)v : -1;
    count[v] = 0;
}

__global__ void cc_union_kernel(const uint8_t *__restrict__ mask, int nx, int ny, int nz,
                                int32_t *parent, int32_t *status) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || !mask[v]) return;
    const int64_t nyz = (int64_t)ny * nz;
    const int ix = (int)(v / nyz);
    const int iy = (int)((v / nz) % ny);
    const int iz = (int)(v % nz);
    if (ix + 1 < nx && mask[v + nyz]) uf_union(parent, (int32_t)v, (int32_t)(v + nyz), status);
    if (iy + 1 < ny && mask[v + nz]) uf_union(parent, (int32_t)v, (int32_t)(v + nz), status);
    if (iz + 1 < nz && mask[v + 1]) uf_union(parent, (int32_t)v, (int32_t)(v + 1), status);
}

__global__ void cc_flatten_kernel(int64_t n, int32_t *parent, int32_t *__restrict__ count,
                                  int32_t *status) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || parent[v] < 0) return;
    const int32_t r = uf_find(parent, (int32_t)v, status);
    parent[v] = r;
    atomicAdd(&count[r], 1);
}

// ------------------------------------------------------------------ breadth-first search
struct BfsArgs {
    int nx, ny, nz;
    int32_t comp_root;
    const double *normals;   // [V, 3]
    const int32_t *root;     // [V] component root or -1
    uint8_t *visited;        // [V]
    unsigned long long *bid; // [V] smallest key bid this level (all-ones: none)
    double *rsdf;            // [V]
    double dx;
};

// direction d: (-x, +y, +x, -y, +z, -z), sdf.py's dX/dY/dZ order
__device__ __forceinline__ bool neighbour(const BfsArgs &a, int32_t v, int d, int32_t &out) {
    const int64_t nyz = (int64_t)a.ny * a.nz;
    const int ix = (int)(v / nyz);
    const int iy = (int)((v / a.nz) % a.ny);
    const int iz = (int)(v % a.nz);
    int jx = ix, jy = iy, jz = iz;
    switch (d) {
        case 0: jx = ix - 1; break;
        case 1: jy = iy + 1; break;
        case 2: jx = ix + 1; break;
        case 3: jy = iy - 1; break;
        case 4: jz = iz + 1; break;
        default: jz = iz - 1; break;
    }
    if (jx < 0 || jy < 0 || jz < 0 || jx >= a.nx || jy >= a.ny || jz >= a.nz) return false;
    out = (int32_t)(((int64_t)jx * a.ny + jy) * a.nz + jz);
    return true;
}

__device__ __forceinline__ bool open_voxel(const BfsArgs &a, int32_t n) {
    return !a.visited[n] && !isnan(a.normals[3 * (int64_t)n]) && a.root[n] == a.comp_root;
}

__global__ void bfs_bid_kernel(const BfsArgs a, const int32_t *__restrict__ frontier, int64_t nf) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf * 6) return;
    int32_t n;
    if (!neighbour(a, frontier[k / 6], (int)(k % 6), n) || !open_voxel(a, n)) return;
    atomicMin(&a.bid[n], (unsigned long long)k);
}

__global__ void bfs_flag_kernel(const BfsArgs a, const int32_t *__restrict__ frontier, int64_t nf,
                                int32_t *__restrict__ flag) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf * 6) return;
    int32_t n;
    int32_t f = 0;
    if (neighbour(a, frontier[k / 6], (int)(k % 6), n) && open_voxel(a, n) &&
        a.bid[n] == (unsigned long long)k)
        f = 1;
    flag[k] = f;
}

// after the exclusive scan pos[k] is the winner's place in the next frontier
__global__ void bfs_emit_kernel(const BfsArgs a, const int32_t *__restrict__ frontier, int64_t nf,
                                const int32_t *__restrict__ pos, int32_t *__restrict__ next) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf * 6) return;
    const int32_t v = frontier[k / 6];
    const int d = (int)(k % 6);
    int32_t n;
    if (!neighbour(a, v, d, n) || !open_voxel(a, n) || a.bid[n] != (unsigned long long)k) return;
    // step * dx as numpy forms it, then dot(): 0 + s0*n0 + s1*n1 + s2*n2 in FP64, in order
    const double sx = d == 0 ? -1.0 : (d == 2 ? 1.0 : 0.0);
    const double sy = d == 1 ? 1.0 : (d == 3 ? -1.0 : 0.0);
    const double sz = d == 4 ? 1.0 : (d == 5 ? -1.0 : 0.0);
    const double *nv = a.normals + 3 * (int64_t)n;
    double acc = 0.0;
    acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sx, a.dx), nv[0]));
    acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sy, a.dx), nv[1]));
    acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sz, a.dx), nv[2]));
    a.rsdf[n] = __dadd_rn(a.rsdf[v], acc);
    next[pos[k]] = n;
}

__global__ void bfs_mark_kernel(const int32_t *__restrict__ next, int64_t n, uint8_t *visited) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) visited[next[k]] = 1;
}

__global__ void bfs_seed_kernel(int32_t seed, int32_t *frontier, uint8_t *visited, double *rsdf) {
    frontier[0] = seed;
    visited[seed] = 1;
    rsdf[seed] = 0.0;
}

// Small frontiers: one CTA runs whole levels -- the same bids, winners, queue positions
// and rsdf values as the per-level kernels above, with __syncthreads between the phases
// instead of kernel boundaries and a host read-back -- until the frontier empties or grows
// past kSmallFrontier entries (then the per-level kernels take over from the frontier it
// leaves in global memory).  Each thread owns a run of consecutive slots k = 6 i + d, so
// a block-wide exclusive scan of the threads' winner counts gives the queue order.  The
// loop ends: every level marks at least one new voxel of a finite component.
constexpr int kSmallThreads = 1024;
constexpr int kSmallFrontier = 4096;  // 24576 slots: at most 24 per thread (one bit each)

struct SmallState {
    int64_t nf;       // frontier size on exit (0: the search is complete)
    int64_t visited;  // voxels marked by this launch
    int32_t parity;   // 1: the exit frontier is in the second buffer
    int32_t pad;
};

__global__ void __launch_bounds__(kSmallThreads) bfs_small_kernel(const BfsArgs a, int32_t *fa,
                                                                  int32_t *fb, int64_t nf0,
                                                                  SmallState *state) {
    __shared__ int32_t warp_tot[kSmallThreads / 32];
    __shared__ int32_t s_total;
    int32_t *cur = fa, *nxt = fb;
    int64_t nf = nf0, marked = 0;
    int32_t parity = 0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    while (nf > 0 && nf <= kSmallFrontier) {
        const int slots = (int)nf * 6;
        const int per = (slots + kSmallThreads - 1) / kSmallThreads;
        const int k0 = tid * per;
        const int k1 = min(k0 + per, slots);
        // bids
        for (int k = k0; k < k1; ++k) {
            int32_t n;
            if (neighbour(a, cur[k / 6], k % 6, n) && open_voxel(a, n))
                atomicMin(&a.bid[n], (unsigned long long)k);
        }
        __syncthreads();
        // winners of this thread's slots
        uint32_t won = 0;
        int32_t cnt = 0;
        for (int k = k0; k < k1; ++k) {
            int32_t n;
            // the bids came from atomics at L2 this level: read them past L1
            if (neighbour(a, cur[k / 6], k % 6, n) && open_voxel(a, n) &&
                __ldcg(&a.bid[n]) == (unsigned long long)k) {
                won |= 1u << (k - k0);
                ++cnt;
            }
        }
        // exclusive scan of the counts over the block, in thread (= slot) order
        int32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int32_t w = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_tot[lane] = w;  // inclusive over warps
            if (lane == 31) s_total = w;
        }
        __syncthreads();
        int32_t pos = incl - cnt + (warp > 0 ? warp_tot[warp - 1] : 0);
        // emit in queue order (the per-level emit kernel's arithmetic)
        for (int k = k0; k < k1; ++k) {
            if (!(won >> (k - k0) & 1u)) continue;
            const int32_t v = cur[k / 6];
            const int d = k % 6;
            int32_t n;
            neighbour(a, v, d, n);
            const double sx = d == 0 ? -1.0 : (d == 2 ? 1.0 : 0.0);
            const double sy = d == 1 ? 1.0 : (d == 3 ? -1.0 : 0.0);
            const double sz = d == 4 ? 1.0 : (d == 5 ? -1.0 : 0.0);
            const double *nv = a.normals + 3 * (int64_t)n;
            double acc = 0.0;
            acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sx, a.dx), nv[0]));
            acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sy, a.dx), nv[1]));
            acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sz, a.dx), nv[2]));
            a.rsdf[n] = __dadd_rn(a.rsdf[v], acc);
            nxt[pos++] = n;
        }
        __syncthreads();
        const int32_t total = s_total;
        for (int i = tid; i < total; i += kSmallThreads) a.visited[nxt[i]] = 1;
        __syncthreads();
        marked += total;
        nf = total;
        int32_t *t = cur;
        cur = nxt;
        nxt = t;
        parity ^= 1;
    }
    if (tid == 0) {
        state->nf = nf;
        state->visited = marked;
        state->parity = parity;
    }
}

// ---------------------------------------------------------------- exclusive int32 scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 1024 values per block

__global__ void scan_block_kernel(int32_t *data, int64_t n, int32_t *block_sums) {
    __shared__ int32_t warp_sums[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    int32_t run = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? data[base + i] : 0;
        const int32_t t = v[i];
        v[i] = run;  // exclusive within the thread
        run += t;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const int32_t offset = (incl - run) + (warp > 0 ? warp_sums[warp - 1] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) data[base + i] = v[i] + offset;
    if (threadIdx.x == kScanThreads - 1) block_sums[blockIdx.x] = offset + run;
}

__global__ void scan_add_kernel(int32_t *data, int64_t n, const int32_t *block_offsets) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) data[k] += block_offsets[k / kScanTile];
}

size_t scan_temp_elems(int64_t n) {
    size_t total = 0;
    while (n > 1) {
        n = (n + kScanTile - 1) / kScanTile;
        total += (size_t)n + 1;
    }
    return total + 2;
}

// exclusive scan of data[0..n) in place; data[n] (one past the end) receives the total
cudaError_t scan_exclusive(int32_t *data, int64_t n, int32_t *temp, cudaStream_t stream) {
    const int64_t blocks = (n + kScanTile - 1) / kScanTile;
    int32_t *sums = temp;
    scan_block_kernel<<<(unsigned)blocks, kScanThreads, 0, stream>>>(data, n, sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (blocks > 1) {
        // scan the block totals (recursively), then add each block's offset
        e = scan_exclusive(sums, blocks, temp + blocks + 1, stream);
        if (e != cudaSuccess) return e;
        scan_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(data, n, sums);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(data + n, sums + blocks, sizeof(int32_t),
                               cudaMemcpyDeviceToDevice, stream);
    }
    return cudaMemcpyAsync(data + n, sums, sizeof(int32_t), cudaMemcpyDeviceToDevice, stream);
}

inline unsigned grid_for(int64_t n, int nt) { return (unsigned)((n + nt - 1) / nt); }

}  // namespace
}  // namespace mmn

using namespace mmn;

namespace {
constexpr size_t kStatus = 256;
inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

bool bad_dims(int32_t nx, int32_t ny, int32_t nz) {
    if (nx < 1 || ny < 1 || nz < 1) return true;
    const int64_t v = (int64_t)nx * ny * nz;
    return v > (int64_t)INT32_MAX / 6;  // flat indices and 6 bids per voxel fit in int32
}
}  // namespace

extern "C" size_t mmn_components_workspace_bytes(int64_t num_voxels) {
    (void)num_voxels;
    return kStatus;
}

extern "C" int mmn_components(int32_t nx, int32_t ny, int32_t nz, const uint8_t *mask,
                              int32_t *root, int32_t *count, void *workspace,
                              size_t workspace_bytes, cudaStream_t stream) {
    if (bad_dims(nx, ny, nz)) return MMN_ERR_INVALID_ARGUMENT;
    if (!mask || !root || !count) return MMN_ERR_NULL_POINTER;
    if (!workspace || workspace_bytes < kStatus ||
        (reinterpret_cast<uintptr_t>(workspace) & 255))
        return MMN_ERR_WORKSPACE;
    const int64_t n = (int64_t)nx * ny * nz;
    int32_t *status = static_cast<int32_t *>(workspace);
    if (cudaMemsetAsync(status, 0, kStatus, stream) != cudaSuccess) return MMN_ERR_CUDA;
    cc_init_kernel<<<grid_for(n, 256), 256, 0, stream>>>(mask, n, root, count);
    cc_union_kernel<<<grid_for(n, 256), 256, 0, stream>>>(mask, nx, ny, nz, root, status);
    cc_flatten_kernel<<<grid_for(n, 256), 256, 0, stream>>>(n, root, count, status);
    return cudaGetLastError() == cudaSuccess ? MMN_OK : MMN_ERR_CUDA;
}

extern "C" size_t mmn_rsdf_workspace_bytes(int32_t nx, int32_t ny, int32_t nz) {
    if (bad_dims(nx, ny, nz)) return 0;
    const int64_t n = (int64_t)nx * ny * nz;
    return kStatus + up256((size_t)n) + up256((size_t)n * 8) + 2 * up256((size_t)n * 4) +
           up256(((size_t)6 * n + 1) * 4) + up256(scan_temp_elems(6 * n) * 4) + 256;
}

extern "C" int mmn_rsdf_component(int32_t nx, int32_t ny, int32_t nz, const double *normals,
                                  const int32_t *root, int32_t comp_root, int32_t seed,
                                  double dx, double *rsdf, int64_t *visited_count,
                                  void *workspace, size_t workspace_bytes,
                                  cudaStream_t stream) {
    if (bad_dims(nx, ny, nz)) return MMN_ERR_INVALID_ARGUMENT;
    if (!normals || !root || !rsdf) return MMN_ERR_NULL_POINTER;
    const int64_t n = (int64_t)nx * ny * nz;
    if (seed < 0 || seed >= n || comp_root < 0 || comp_root >= n || !(dx > 0.0))
        return MMN_ERR_INVALID_ARGUMENT;
    const size_t need = mmn_rsdf_workspace_bytes(nx, ny, nz);
    if (!workspace || workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255))
        return MMN_ERR_WORKSPACE;
    unsigned char *w = static_cast<unsigned char *>(workspace);
    size_t off = kStatus;
    uint8_t *visited = w + off;
    off += up256((size_t)n);
    unsigned long long *bid = reinterpret_cast<unsigned long long *>(w + off);
    off += up256((size_t)n * 8);
    int32_t *fa = reinterpret_cast<int32_t *>(w + off);
    off += up256((size_t)n * 4);
    int32_t *fb = reinterpret_cast<int32_t *>(w + off);
    off += up256((size_t)n * 4);
    int32_t *flag = reinterpret_cast<int32_t *>(w + off);
    off += up256(((size_t)6 * n + 1) * 4);
    int32_t *temp = reinterpret_cast<int32_t *>(w + off);

    if (cudaMemsetAsync(w, 0, kStatus, stream) != cudaSuccess ||
        cudaMemsetAsync(visited, 0, (size_t)n, stream) != cudaSuccess ||
        cudaMemsetAsync(bid, 0xff, (size_t)n * 8, stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    BfsArgs a;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.comp_root = comp_root;
    a.normals = normals;
    a.root = root;
    a.visited = visited;
    a.bid = bid;
    a.rsdf = rsdf;
    a.dx = dx;
    bfs_seed_kernel<<<1, 1, 0, stream>>>(seed, fa, visited, rsdf);
    int64_t nf = 1, total = 1;
    // the single-CTA search's exit state, in the workspace header after the status word
    SmallState *small = reinterpret_cast<SmallState *>(w + 64);
    // every level (and every single-CTA launch) adds at least one voxel, so n rounds bound
    // the search
    for (int64_t level = 0; nf > 0 && level <= n; ++level) {
        if (nf <= kSmallFrontier) {
            bfs_small_kernel<<<1, kSmallThreads, 0, stream>>>(a, fa, fb, nf, small);
            SmallState hs;
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(&hs, small, sizeof(hs), cudaMemcpyDeviceToHost, stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess)
                return MMN_ERR_CUDA;
            total += hs.visited;
            nf = hs.nf;
            if (hs.parity) {
                int32_t *t = fa;
                fa = fb;
                fb = t;
            }
            continue;
        }
        const int64_t slots = nf * 6;
        bfs_bid_kernel<<<grid_for(slots, 256), 256, 0, stream>>>(a, fa, nf);
        bfs_flag_kernel<<<grid_for(slots, 256), 256, 0, stream>>>(a, fa, nf, flag);
        if (scan_exclusive(flag, slots, temp, stream) != cudaSuccess) return MMN_ERR_CUDA;
        bfs_emit_kernel<<<grid_for(slots, 256), 256, 0, stream>>>(a, fa, nf, flag, fb);
        int32_t next_n = 0;
        if (cudaMemcpyAsync(&next_n, flag + slots, sizeof(int32_t), cudaMemcpyDeviceToHost,
                            stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return MMN_ERR_CUDA;
        if (next_n > 0)
            bfs_mark_kernel<<<grid_for(next_n, 256), 256, 0, stream>>>(fb, next_n, visited);
        if (cudaGetLastError() != cudaSuccess) return MMN_ERR_CUDA;
        nf = next_n;
        total += next_n;
        int32_t *t = fa;
        fa = fb;
        fb = t;
    }
    if (visited_count) *visited_count = total;
    int32_t st = 0;
    if (cudaMemcpyAsync(&st, w, sizeof(int32_t), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return MMN_ERR_CUDA;
    return st ? st : MMN_OK;
}

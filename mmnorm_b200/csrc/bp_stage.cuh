// bp_stage.cuh -- device helpers shared by the forward and backward kernels: the
// double-buffered shared-memory antenna stage filled by bulk TMA copies, and voxel
// index decoding / result stores.
#pragma once
#include "bp_kernels.cuh"

namespace mmn {

// After a bounded wait on chunk `gc` of a double-buffered stage gave up: the issuing thread
// gives each stage that may still have a copy outstanding -- chunk gc, and chunk gc+1 when
// it was issued -- one more bounded wait, so that a copy which is merely late lands before
// the CTA exits and its shared memory can go to another CTA.  A copy that misses this wait
// too may still be in flight when the CTA exits.  Called by every thread of the CTA; not
// inlined, so that the failure path stays out of the kernels' register allocation.
static __device__ __noinline__ void drain_stages(uint64_t *bars, uint32_t gc, bool next_issued,
                                                 int32_t *status) {
    if (threadIdx.x == 0) {
        mbar_wait_bounded(&bars[gc & 1], (gc >> 1) & 1, status);
        if (next_issued) mbar_wait_bounded(&bars[(gc + 1) & 1], ((gc + 1) >> 1) & 1, status);
    }
    __syncthreads();
}

// ----------------------------------------------------------- shared-memory stage
struct Stage {
    uint64_t *bars;
    unsigned char *base;
    size_t stage_bytes;
    int nas;
    int esz;  // bytes per sample in shared memory (8: (re, im); 16: (re, re, im, im))
    int fp;

    // Fill stage buffer `s` with chunk `c` (antennas a_begin + c*nas ...) of a work item.
    __device__ void issue(const FwdParams &p, int c, int s, int a_begin, int a_end) const {
        const int a0 = a_begin + c * nas;
        const int na = min(nas, a_end - a0);
        unsigned char *st = base + s * stage_bytes;
        const uint32_t ant_bytes = (uint32_t)(na * sizeof(AntRec));
        const uint32_t meas_bytes = (uint32_t)((size_t)na * fp * esz);
        unsigned char *mdst = st + (size_t)nas * sizeof(AntRec);
        const unsigned char *msrc =
            static_cast<const unsigned char *>(p.meas) + (size_t)a0 * fp * esz;
        // A bulk copy needs 16-byte aligned addresses and a size that is a multiple of 16
        // bytes; a layout that breaks this is refused here (status word, barrier completed
        // with no bytes) instead of faulting the copy engine.
        if (((uintptr_t)st | (uintptr_t)mdst | (uintptr_t)msrc |
             (uintptr_t)(p.ant + a0) | ant_bytes | meas_bytes) & 15u) {
            set_status(p.status, MMN_ERR_INVALID_ARGUMENT);
            mbar_arrive(&bars[s]);
            return;
        }
        mbar_arrive_expect_tx(&bars[s], ant_bytes + meas_bytes);
        bulk_g2s(st, p.ant + a0, ant_bytes, &bars[s]);
        bulk_g2s(mdst, msrc, meas_bytes, &bars[s]);
    }
    __device__ void issue(const FwdParams &p, int c, int a_begin, int a_end) const {
        issue(p, c, c & 1, a_begin, a_end);
    }
    // Called by every thread after a bounded wait on chunk `gc` gave up (the status word
    // is set): see drain_stages.
    __device__ void drain_after_timeout(uint32_t gc, bool next_issued, int32_t *status) const {
        drain_stages(bars, gc, next_issued, status);
    }
    __device__ const AntRec *ants(int s) const {
        return reinterpret_cast<const AntRec *>(base + s * stage_bytes);
    }
    __device__ const unsigned char *meas(int s) const {
        return base + s * stage_bytes + (size_t)nas * sizeof(AntRec);
    }
};

__device__ __forceinline__ void decode_voxel(const FwdParams &p, int64_t rel, float &x,
                                             float &y, float &z) {
    const int64_t v = rel < p.vox_count ? p.vox_start + rel : p.vox_start;
    const int64_t nyz = (int64_t)p.ny * p.nz;
    const int ix = (int)(v / nyz);
    const int64_t rem = v - (int64_t)ix * nyz;
    const int iy = (int)(rem / p.nz);
    const int iz = (int)(rem - (int64_t)iy * p.nz);
    x = __ldg(p.x_locs + ix);
    y = __ldg(p.y_locs + iy);
    z = __ldg(p.z_locs + iz);
}

__device__ __forceinline__ void store_voxel(const FwdParams &p, int split, int64_t rel,
                                            const float (&a)[8]) {
    if (rel >= p.vox_count) return;
    const int64_t v = p.vox_start + rel;
    if (p.num_splits == 1) {
        if (p.image) p.image[v] = make_float2(a[0], a[1]);
        if (p.out_r) {
            p.out_r[v] = a[0];
            p.out_i[v] = a[1];
        }
        if (p.vote) {
            p.vote[v] = make_float2(a[2], a[3]);
            p.vote[p.nvox + v] = make_float2(a[4], a[5]);
            p.vote[2 * p.nvox + v] = make_float2(a[6], a[7]);
        }
    } else {
        float4 *dst = p.partial + 2 * ((size_t)split * p.vox_count + rel);
        dst[0] = make_float4(a[0], a[1], a[2], a[3]);
        dst[1] = make_float4(a[4], a[5], a[6], a[7]);
    }
}


}  // namespace mmn

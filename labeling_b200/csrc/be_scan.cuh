// be_scan.cuh -- the segment-count scan shared by the 2D and 3D pipelines.
//
// Segment counts are uint8 (at most half a segment's pixels can start a component).  The scan
// runs in two launches: k_post_* sums each chunk of kScanChunk counts (chunk_sum below) while it
// ranks border roots, and k_segscan turns the counts into an exclusive uint32 prefix.
#pragma once
#include "be_common.cuh"

namespace be {

// Sum of segcnt[c * kScanChunk, ...) into w.chunksum[c]; called by a whole CTA.
template <int NT>
__device__ __forceinline__ void chunk_sum(Work &w, int64_t c, uint32_t *tmp)
{
    const int64_t lo = c * kScanChunk, hi = min(w.n_segs, lo + kScanChunk);
    uint32_t s = 0;
    for (int64_t i = lo + int64_t(threadIdx.x) * 16; i < hi; i += int64_t(NT) * 16) {
        if (i + 16 <= hi) {
            const uint4 v = *reinterpret_cast<const uint4 *>(w.segcnt + i);
            s += __vsadu4(v.x, 0u) + __vsadu4(v.y, 0u) + __vsadu4(v.z, 0u) + __vsadu4(v.w, 0u);
        } else {
            for (int64_t k = i; k < hi; ++k) s += w.segcnt[k];
        }
    }
    uint32_t total;
    block_exscan<NT>(s, tmp, &total);
    if (threadIdx.x == 0) w.chunksum[c] = total;
}

}  // namespace be

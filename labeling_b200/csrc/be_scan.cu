// be_scan.cu -- exclusive scan of the per-segment root counts for the iterative forms: k_chunk_sums
// sums each chunk, k_segscan scans them (the union-find pipelines use the single-pass scan of
// be_scan.cuh inside their scan + node launch).
#include "be_kernels.h"
#include "be_scan.cuh"

namespace be {

// One CTA per chunk of kScanChunk segments: adds the sums of all earlier chunks, scans its own
// counts and writes segpref[i] = sum of segcnt[0, i).  The last chunk also writes segpref[n_segs].
__global__ void __launch_bounds__(kScanThreads) k_segscan(Work w)
{
    // The release comes after the wait on purpose: the label-write launch that follows reads the
    // post-merge pass's results before its own wait, which is safe only because this grid lets it
    // start once that pass has completed.
    grid_dep_wait();
    grid_dep_release();
    constexpr int NT = kScanThreads;
    constexpr int PER = kScanChunk / NT;   // 16 counts per thread
    __shared__ uint32_t tmp[NT / 32 + 1];
    const int64_t c = blockIdx.x;
    uint32_t off = 0;
    for (int64_t k = threadIdx.x; k < c; k += NT) off += w.chunksum[k];
    uint32_t total;
    block_exscan<NT>(off, tmp, &total);
    off = total;

    const int64_t lo = c * kScanChunk + int64_t(threadIdx.x) * PER;
    const int64_t hi = min(w.n_segs, lo + PER);
    uint32_t v[PER / 4];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < PER / 4; ++q) {
        const int64_t i = lo + 4 * q;
        uint32_t x = 0;
        if (i + 4 <= hi) {
            x = *reinterpret_cast<const uint32_t *>(w.segcnt + i);
        } else {
            for (int k = 0; k < 4; ++k)
                if (i + k < hi) x |= uint32_t(w.segcnt[i + k]) << (8 * k);
        }
        v[q] = x;
        s += __vsadu4(x, 0u);
    }
    uint32_t ctot;
    uint32_t pre = off + block_exscan<NT>(s, tmp, &ctot);
#pragma unroll
    for (int q = 0; q < PER / 4; ++q) {
        const int64_t i = lo + 4 * q;
        uint4 o;
        o.x = pre; pre += v[q] & 0xFF;
        o.y = pre; pre += (v[q] >> 8) & 0xFF;
        o.z = pre; pre += (v[q] >> 16) & 0xFF;
        o.w = pre; pre += v[q] >> 24;
        if (i + 4 <= hi) {
            *reinterpret_cast<uint4 *>(w.segpref + i) = o;
        } else {
            if (i < hi) w.segpref[i] = o.x;
            if (i + 1 < hi) w.segpref[i + 1] = o.y;
            if (i + 2 < hi) w.segpref[i + 2] = o.z;
        }
    }
    if (c == gridDim.x - 1 && threadIdx.x == 0) w.segpref[w.n_segs] = off + ctot;
}

// Chunk sums (one CTA per chunk), the first half of the two-launch scan.
__global__ void __launch_bounds__(kPostThreads) k_chunk_sums(Work w)
{
    __shared__ uint32_t tmp[kPostThreads / 32 + 1];
    chunk_sum<kPostThreads>(w, blockIdx.x, tmp);
}

}  // namespace be

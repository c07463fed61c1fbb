// be_scan.cuh -- the segment-count scan and the node-link pass shared by the 2D and 3D pipelines.
//
// Segment counts are uint8 (at most half a segment's pixels can start a component).  The
// union-find pipelines scan them in one launch (segscan_lb_chunk, a single-pass scan with a
// decoupled look-back) beside the node pass (flatten_tile_nodes in 2D, link_tile_nodes in 3D);
// the iterative forms use the two-launch scan of be_scan.cu (k_chunk_sums with chunk_sum below,
// then k_segscan).
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

// Single-pass scan of the segment counts (decoupled look-back): one CTA per chunk of kScanChunk
// segments, chunks taken in the order the CTAs start (a ticket), so every chunk a CTA looks back at
// belongs to a CTA that started earlier and publishes without waiting on anyone.  A chunk publishes
// its own sum first, then its inclusive prefix once it knows its exclusive one; a status word is
// (epoch << 34) | (state << 32) | value, and only words of this run's epoch count, so the words
// never need clearing between runs.  Waits are bounded: a wait that runs out sets w.err[3] and the
// chunk goes on with what it has (the labels are then wrong, the device stays usable).
// Called by a whole CTA of NT threads; tmp holds NT / 32 + 1 words, sh two.
template <int NT>
__device__ __forceinline__ void segscan_lb_chunk(Work &w, uint32_t *tmp, uint32_t *sh)
{
    constexpr int PER = kScanChunk / NT;
    constexpr uint32_t kSpinCap = 1u << 17;   // well over any real wait, a fraction of a second
    uint32_t &sh_c = sh[0], &sh_excl = sh[1];
    if (threadIdx.x == 0) sh_c = atomicAdd(w.epoch + 1, 1u);
    __syncthreads();
    const int64_t c = sh_c;
    const uint64_t ep = uint64_t(ld_volatile(w.epoch)) & 0x3FFFFFFFull;

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
    uint32_t pre = block_exscan<NT>(s, tmp, &ctot);
    volatile unsigned long long *st = reinterpret_cast<volatile unsigned long long *>(w.scan_status);
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        if (lane == 0) st[c] = (ep << 34) | (1ull << 32) | ctot;   // this chunk's sum
        // Look back 32 chunks at a time: lane k reads chunk c - 1 - k - base.
        uint32_t excl = 0;
        int64_t base = 0;
        uint32_t spins = 0;
        while (c - 1 - base >= 0) {
            const int64_t j = c - 1 - base - lane;
            uint64_t sw = 0;
            uint32_t state = 2;   // chunks before 0 count as an empty inclusive prefix
            if (j >= 0) {
                sw = st[j];
                state = (sw >> 34) == ep ? uint32_t(sw >> 32) & 3u : 0u;
            }
            const uint32_t incl = __ballot_sync(0xFFFFFFFFu, state == 2);
            const uint32_t unready = __ballot_sync(0xFFFFFFFFu, state == 0);
            // Only the chunks up to the nearest inclusive prefix matter (all 32 when none is).
            const uint32_t need = incl ? ((2u << (__ffs(incl) - 1)) - 1u) : 0xFFFFFFFFu;
            if (unready & need) {
                if (++spins > kSpinCap) {   // cannot happen while the scheduler runs earlier CTAs
                    if (lane == 0) atomicExch(w.err + 3, 1u);
                    break;
                }
                continue;
            }
            // Sum back to (and including) the nearest inclusive prefix among the 32.
            const int stop = __ffs(incl) - 1;   // lowest lane = nearest chunk
            uint32_t val = (j >= 0 && lane <= (incl ? stop : 31)) ? uint32_t(sw) : 0u;
#pragma unroll
            for (int o = 16; o; o >>= 1) val += __shfl_xor_sync(0xFFFFFFFFu, val, o);
            excl += val;
            if (incl) break;
            base += 32;
        }
        if (lane == 0) {
            st[c] = (ep << 34) | (2ull << 32) | uint32_t(excl + ctot);   // inclusive prefix
            sh_excl = excl;
        }
    }
    __syncthreads();
    pre += sh_excl;
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
    if (c == w.n_chunks - 1 && threadIdx.x == 0) w.segpref[w.n_segs] = sh_excl + ctot;
}

// Points every linked node of tile t at its global root (gfind_jump: the nodes of all tiles jump
// at once, each writing only its own entry, so deep trees take logarithmic walks).  Called by a
// whole CTA.
__device__ __forceinline__ void flatten_tile_nodes(Work &w, int64_t t, int maxb)
{
    const uint32_t nb = w.nb[t];
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const uint32_t node = uint32_t(t * maxb + j);
        if (uint32_t(w.gp[node]) == node) continue;
        const uint32_t root = gfind_jump(w.gp, node);
        w.gp[node] = w.gp[root];
    }
}

// As flatten_tile_nodes, and resolves each node's link for the label writes: nlink[node] =
// (segment of the root's first pixel, (node's root block << 16) | rank of that pixel among the
// roots left in its segment), or x = kNone for a node that is a root.  locate(key, &seg, &rank)
// finds the segment and the rank of the pixel with raster key `key` from the root bitmaps, which
// the merge has left final.  Called by a whole CTA.
template <typename Locate>
__device__ __forceinline__ void link_tile_nodes(Work &w, int64_t t, int maxb, Locate locate)
{
    const uint32_t nb = w.nb[t];
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const uint32_t node = uint32_t(t * maxb + j);
        uint2 link = make_uint2(kNone, 0u);
        if (uint32_t(w.gp[node]) != node) {
            const uint32_t root = gfind_jump(w.gp, node);
            const unsigned long long re = w.gp[root];
            w.gp[node] = re;
            uint32_t seg, rank;
            locate(uint32_t(re >> 32), seg, rank);
            link = make_uint2(seg, (uint32_t(w.nroot[node]) << 16) | rank);
        }
        w.nlink[node] = link;
    }
}

}  // namespace be

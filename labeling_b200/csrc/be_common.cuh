// be_common.cuh -- shared device code for the B200 Block-Equivalence labeler.
//
// Terminology (follows the reference's BE method, LabelingAlgs.cl:133-319 / 737-979):
//   block      2x2 pixels (2D) or 2x2x2 voxels (3D); the reference's "super pixel".
//   mask       which pixels/voxels of a block are foreground (4 / 8 bits).
//   tile       the rectangle (box) of blocks one CTA labels in shared memory.
//   key        the raster index of a pixel/voxel inside its image (row-major, last dim fastest).
//              A component is represented by its smallest key (its first pixel in raster order);
//              that is what makes the output canonical.
//   node       a tile-local component that touches the tile border; nodes are merged across
//              tiles with a global union-find.
//   segment    the part of one image row (a line along the fastest dimension) that lies in one
//              tile; per-segment root counts give each component its canonical rank.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

namespace be {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------------------------
// Image descriptors.  One pipeline launch labels a list of images (the plain API passes one).
// ---------------------------------------------------------------------------------------------
struct Img2D {
    const uint8_t *in;   // row-major uint8, in_pitch bytes per row
    int32_t *out;        // row-major int32 labels, out_pitch elements per row
    int64_t in_pitch;
    int64_t out_pitch;
    int32_t rows, cols;
    int32_t tiles_x, tiles_y;
    int64_t tile_base;   // index of the image's first tile in the launch
    int64_t seg_base;    // index of the image's first segment in the launch
    int32_t thr;         // foreground is pixel > thr
    int32_t index;       // position in the caller's list (for per-image outputs)
};

struct Img3D {
    const uint8_t *in;   // dense [d0][d1][d2] uint8, d2 fastest
    int32_t *out;        // dense [d0][d1][d2] int32 labels
    int32_t d0, d1, d2;
    int32_t t0, t1, t2;  // tile counts per dimension
    int64_t tile_base;
    int64_t seg_base;
    int32_t thr;
    int32_t index;
};

// The images of one launch: a device array, or a single descriptor passed by value (plain calls
// need no descriptor upload).
template <class Img>
struct ImgList {
    const Img *ptr;
    int n;
    Img one;
    __device__ __forceinline__ Img get(int64_t tile) const;
};

// Global scratch of one pipeline launch ("workspace").  Sizes are per tile so that every tile
// owns fixed-size slices and no kernel needs a prefix sum to find its data.
struct Work {
    void *lab;            // per-block tile-local labels: uint16 (2D) / uint32 (3D), NBLK per tile
    uint16_t *perim;      // per tile NPERIM border entries: (node << 4) | side bits, 0 = empty
    uint32_t *nb;         // per tile: number of nodes
    unsigned long long *gp;   // per node (tile * MAXB + j): union-find entry (key of the parent << 32) |
                              // parent (global node id); see gentry
    uint16_t *nroot;      // per node: tile-local block index of the node's root block
    uint2 *nlink;         // per node, after the merge: x = segment of its global root's first pixel
                          // (kNone when the node is a root itself), y = (root block << 16) | rank
                          // of that first pixel among the roots left in its segment
    uint32_t *rbits;      // per tile: bitmap of the first pixels (voxels) of the tile's components
                          // that are still roots (the merge clears the ones it links)
    uint8_t *segcnt;      // per segment: number of component roots (uint8, word-padded)
    uint32_t *segpref;    // per segment + 1: exclusive prefix of segcnt over the launch
    uint32_t *chunksum;   // per scan chunk: sum of segcnt
    uint32_t *queue;      // work-queue counters (persistent mode); zeroed before a launch
    int64_t *ncomp;       // per image: number of components
    uint32_t *err;        // error flags (bounded waits / iteration caps)
    uint32_t *epoch;      // [0] launch epoch (+1 per pipeline run), [1] scan ticket counter
    uint64_t *scan_status;  // per scan chunk: (epoch << 34 | state << 32) | prefix value
    int64_t n_tiles;
    int64_t n_segs;
    int32_t n_chunks;
    int32_t n_imgs;
};

constexpr int kScanChunk = 4096;    // segments per scan chunk (one CTA)

// ---------------------------------------------------------------------------------------------
// Bounds-checked build (-DBE_BOUNDS_CHECK): GUARD(w, cond, site, value) is false when `cond`
// fails; the first failure of a launch records (site, value) in w.err[0..2] and the guarded
// access is skipped.  In normal builds GUARD is the constant true and costs nothing.
// ---------------------------------------------------------------------------------------------
#ifdef BE_BOUNDS_CHECK
__device__ __forceinline__ bool be_guard(uint32_t *err, bool ok, uint32_t site, uint64_t val)
{
    if (!ok && atomicCAS(err, 0u, site) == 0u) {
        err[1] = uint32_t(val);
        err[2] = uint32_t(val >> 32);
    }
    return ok;
}
#define GUARD(w, cond, site, val) be_guard((w).err, bool(cond), (site), uint64_t(val))
#else
#define GUARD(w, cond, site, val) (true)
#endif

// ---------------------------------------------------------------------------------------------
// Small helpers.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p)
{
    return *reinterpret_cast<const volatile uint32_t *>(p);
}

// Foreground bits of four packed pixels: bit k = byte k > thr.
__device__ __forceinline__ uint32_t fg4(uint32_t w, uint32_t thr4)
{
    uint32_t m = __vcmpgtu4(w, thr4) & 0x01010101u;
    return (m * 0x10204080u) >> 28;
}

// Foreground bits of 16 pixels held in a uint4 (bit k = pixel k).
__device__ __forceinline__ uint32_t fg16(uint4 v, uint32_t thr4)
{
    return fg4(v.x, thr4) | (fg4(v.y, thr4) << 4) | (fg4(v.z, thr4) << 8) | (fg4(v.w, thr4) << 12);
}

// Spread the 8 bit-pairs of a 16-bit word into the low two bits of 8 nibbles.
__device__ __forceinline__ uint32_t pairs_to_nibbles(uint32_t x)
{
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    return x;
}

// Union-find find over a shared-memory parent array (parents never exceed their child), with
// path halving: each visited entry is pointed at its grandparent.  Every stored value is an
// ancestor of the entry at the time it was read, so concurrent merges stay correct: a pointer
// never leaves the entry's component, and a merge that loses a race to such a store retries
// from the parent it displaced (see smerge).
__device__ __forceinline__ uint32_t sfind(uint32_t *P, uint32_t a)
{
    uint32_t p = P[a];
    while (p != a) {
        const uint32_t g = P[p];
        if (g != p) P[a] = g;
        a = p;
        p = g;
    }
    return a;
}

// Find without writes, for the flatten pass after all merges: no link can happen any more, so the
// entry reached is the true root.  (Path halving is not allowed there: a halving store that lands
// after the entry's owner wrote its root would point the entry back at an inner node.)
__device__ __forceinline__ uint32_t sfind_ro(const uint32_t *P, uint32_t a)
{
    uint32_t p = P[a];
    while (p != a) {
        a = p;
        p = P[a];
    }
    return a;
}

// Root of `a` after all merges, pointing every entry on the path straight at it.  Safe while
// other threads do the same: all of them store the same final root into shared entries.
__device__ __forceinline__ uint32_t sflatten(uint32_t *P, uint32_t a)
{
    const uint32_t r = sfind_ro(P, a);
    uint32_t x = a;
    while (x != r) {
        const uint32_t nx = P[x];
        P[x] = r;
        x = nx;
    }
    return r;
}

// Merge of two shared-memory union-find trees that keeps the smaller index as the root
// (the atomicMin formulation of Playne & Hawick's union-find, safe under concurrent merges).
__device__ __forceinline__ void smerge(uint32_t *P, uint32_t a, uint32_t b)
{
    for (;;) {
        a = sfind(P, a);
        b = sfind(P, b);
        if (a == b) return;
        if (a < b) {
            uint32_t old = atomicMin(&P[b], a);
            if (old == b) return;
            b = old;
        } else {
            uint32_t old = atomicMin(&P[a], b);
            if (old == a) return;
            a = old;
        }
    }
}

// Appends this lane's `n` merge pairs to a shared queue with one atomic per warp; returns the
// lane's first position (positions >= capacity mean the queue is full for those pairs).
__device__ __forceinline__ uint32_t warp_reserve(uint32_t *count, uint32_t n)
{
    const int lane = threadIdx.x & 31;
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    uint32_t base = 0;
    if (lane == 31 && total) base = atomicAdd(count, total);
    base = __shfl_sync(0xFFFFFFFFu, base, 31);
    return base + incl - n;
}

// Global union-find entries: gp[x] = (key of x's parent << 32) | parent, a root holding its own key
// and index.  Keys (first-pixel raster indices) are distinct, and a parent's key is always smaller
// than its child's, so no path can close a cycle whatever other threads link meanwhile, and one
// load of an entry gives both the parent and the key that decides which way a union goes.
__device__ __forceinline__ unsigned long long gentry(uint32_t key, uint32_t id)
{
    return (static_cast<unsigned long long>(key) << 32) | id;
}

// Union of nodes a and b after Rem's algorithm, lock-free: the two sides climb in turn, always
// the side whose parent has the larger key (the order keys are linked in), with path halving on
// the way; the walk ends where the two parents meet (already one set), or when the climbing side
// stands on a root, which is linked (CAS) under the other side's parent -- a node of b's set with
// a smaller key.  A walk that reaches the common ancestor stops there instead of going on to both
// roots.  Latency, not work, is the cost: each step is one L2 round trip, and one load gives the
// parent and its key.  on_link(key) is called with the key of the root that was linked.  (Rem's
// splicing -- re-pointing the climbing node at the other side's parent -- was measured: it merged
// the long paths of one-pixel spirals into deep trees.)
template <typename OnLink>
__device__ __forceinline__ void gunion_keyed(unsigned long long *gp, uint32_t a, uint32_t b, OnLink on_link)
{
    volatile unsigned long long *vp = gp;
    unsigned long long ea = vp[a], eb = vp[b];
    for (;;) {
        if (uint32_t(ea) == uint32_t(eb)) return;   // same parent: one set
        if ((ea >> 32) < (eb >> 32)) {               // climb on the side with the larger parent key
            const uint32_t t = a; a = b; b = t;
            const unsigned long long u = ea; ea = eb; eb = u;
        }
        const uint32_t pa = uint32_t(ea);
        if (pa == a) {   // a root
            const unsigned long long old = atomicCAS(gp + a, ea, eb);
            if (old == ea) {
                on_link(uint32_t(ea >> 32));
                return;
            }
            ea = old;
            eb = vp[b];
            continue;
        }
        const unsigned long long ga = vp[pa];
        if (uint32_t(ga) != pa) vp[a] = ga;   // halving
        a = pa;
        ea = ga;
    }
}

// Find with path halving after all merges of the launch are complete: no link can happen any more,
// so every pointer stored is to an ancestor and any interleaving of the stores keeps the trees
// valid.  The cap only bounds the walk should the forest ever hold a cycle (it cannot).
__device__ __forceinline__ uint32_t gfind_halve(unsigned long long *gp, uint32_t a)
{
    volatile unsigned long long *vp = gp;
    unsigned long long e = vp[a];
    for (int it = 0; uint32_t(e) != a && it < (1 << 24); ++it) {
        const uint32_t p = uint32_t(e);
        const unsigned long long g = vp[p];
        if (uint32_t(g) != p) vp[a] = g;
        a = p;
        e = g;
    }
    return a;
}

// Root of node x after all merges of the launch are complete, by pointer jumping that writes only
// x's own entry: each step x is pointed at its parent's parent as that entry reads now.  When every
// node of a deep tree runs this at once, each read lands on an entry that its own thread has
// already shortened, so the walks take about log2(depth) steps instead of depth (and no two
// threads write the same entry).  The cap only bounds the walk should the forest ever hold a cycle
// (it cannot).
__device__ __forceinline__ uint32_t gfind_jump(unsigned long long *gp, uint32_t x)
{
    volatile unsigned long long *vp = gp;
    uint32_t p = uint32_t(vp[x]);
    if (p == x) return x;
    for (int it = 0; it < (1 << 24); ++it) {
        const unsigned long long ep = vp[p];
        const uint32_t g = uint32_t(ep);
        if (g == p) break;   // p is the root
        vp[x] = ep;
        p = g;
    }
    return p;
}

// ---- Border-merge filter ---------------------------------------------------------------------
// The cross-tile merge kernels see the same pair of border components over and over (every face
// position of a large component yields one).  Before a pair costs a global union (dependent loads
// through L2), it is merged in a small shared-memory union-find over the tile's nodes and the
// staged neighbour positions: only a pair that joins two different local sets goes on to the
// global union-find; a pair already connected by earlier local merges is implied by the global
// unions those merges queued.
// Local merge of the sets of slots a and b (smaller slot wins, as smerge); false only when the
// two were already one set and this call changed no parent.  An atomicMin that lands on an entry
// another thread has just linked still rewrites that entry's parent (it moves the entry's subtree
// under `a`), so a call that changed anything reports true: every local link then has a pair
// that goes on to the global union-find, and local connectivity never runs ahead of the global.
__device__ __forceinline__ bool smerge_joined(uint32_t *P, uint32_t a, uint32_t b)
{
    bool changed = false;
    for (;;) {
        a = sfind(P, a);
        b = sfind(P, b);
        if (a == b) return changed;
        if (a < b) {
            const uint32_t old = atomicMin(&P[b], a);
            if (old == b) return true;
            changed |= old > a;
            b = old;
        } else {
            const uint32_t old = atomicMin(&P[a], b);
            if (old == a) return true;
            changed |= old > b;
            a = old;
        }
    }
}

// Decrement a uint8 counter packed in a 32-bit word (the counter is >= 1 when this is called).
__device__ __forceinline__ void dec_u8(uint8_t *base, int64_t idx)
{
    uint32_t *w = reinterpret_cast<uint32_t *>(base + (idx & ~int64_t(3)));
    atomicSub(w, 1u << (8 * (idx & 3)));
}

// Block-wide exclusive scan of one uint32 per thread; returns the thread's prefix and writes the
// total to *total.  `tmp` must hold blockDim.x / 32 + 1 words.
template <int NT>
__device__ __forceinline__ uint32_t block_exscan(uint32_t v, uint32_t *tmp, uint32_t *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < NT / 32 ? tmp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < NT / 32) tmp[lane] = s;
        if (lane == NT / 32 - 1) tmp[NT / 32] = s;
    }
    __syncthreads();
    uint32_t r = x - v + (warp ? tmp[warp - 1] : 0);
    *total = tmp[NT / 32];
    __syncthreads();
    return r;
}

// Index of the image that owns global item `t`, by binary search over the images' bases.
template <class Img>
__device__ __forceinline__ int find_img_tile(const Img *imgs, int n, int64_t t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (imgs[mid].tile_base <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class Img>
__device__ __forceinline__ Img ImgList<Img>::get(int64_t tile) const
{
    return n == 1 ? one : ptr[find_img_tile(ptr, n, tile)];
}

using ImgList2D = ImgList<Img2D>;
using ImgList3D = ImgList<Img3D>;

// Programmatic dependent launch (sm_90 and later).  A launch made with programmatic stream
// serialization may put its CTAs on the SMs while the grid before it in the stream still runs:
// grid_dep_wait() blocks until that grid has completed and its writes are visible (for a normal
// launch it returns at once), and grid_dep_release() lets the next grid's CTAs be scheduled once
// every CTA of this grid has called it or exited.  The pipeline kernels wait before their first
// global access, so the overlap only hides launch and ramp-up time, never a dependency.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Asynchronous global -> shared copies (cp.async, through L1): the data lands in shared memory
// without passing through registers, so a CTA can fetch its next tile's small arrays while it
// works on the current one.  cp_async_wait() waits for all of this thread's copies; a barrier
// after it makes every thread's copies visible to the CTA.
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)   // L2 only
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Launches kernel k, with programmatic stream serialization when `overlap` is set.
template <typename... P, typename... A>
inline cudaError_t launch_k(void (*k)(P...), unsigned grid, unsigned block, cudaStream_t s, bool overlap,
                            A &&...args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = overlap ? 1u : 0u;
    return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// Work distribution: with a queue counter every CTA pulls items until none are left (persistent
// launch); without one, CTA b takes items b, b + grid, ...
struct ItemLoop {
    uint32_t *queue;
    int64_t n;
    __device__ __forceinline__ int64_t first(uint32_t *slot)
    {
        if (!queue) return blockIdx.x;
        if (threadIdx.x == 0) *slot = atomicAdd(queue, 1u);
        __syncthreads();
        int64_t v = *slot;
        __syncthreads();
        return v;
    }
    __device__ __forceinline__ int64_t next(int64_t cur, uint32_t *slot)
    {
        if (!queue) return cur + gridDim.x;
        return first(slot);
    }
};

}  // namespace be

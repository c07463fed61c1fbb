// be_slab.cu -- slab split of one image: label each slab on its own, then join the slabs in one
// exchange step.
//
// A slab is a band of consecutive rows of a 2D image, or of consecutive planes along d0 (the
// slowest dimension) of a volume.  Each slab is labeled by be_label2d / be_label3d on its own --
// on its own GPU, or one after another on one GPU -- which numbers its components 1..K_s in the
// raster order of their first pixels within the slab.  The exchange step needs only each slab's
// first and last row (plane) of labels and its count K_s:
//
//   be_slab_merge    (host) unions the pieces that touch across every slab border -- a pixel of
//                    one slab's last row and a pixel of the next slab's first row in one of the
//                    three columns around it (8-connectivity), or a voxel of the last plane and one
//                    of the nine voxels around it in the next slab's first plane (26-connectivity)
//                    -- and derives every slab's label map;
//   be_slab_relabel  (device) applies one slab's map to its labels in place.
//
// Canonical numbering carries over.  The raster order of the whole image orders pieces by slab,
// then by local label (slab s lies before slab s + 1, and within a slab the local labels are in
// first-pixel order), so a component's first pixel is the first pixel of its piece with the
// smallest key (slab, local label).  Unions keep that piece as the root.  A piece that is joined
// under an earlier piece takes the root's label; a root piece (s, l) gets
//
//     offset_s + l - (joined pieces of slab s with a local label below l),
//
// offset_s = the root pieces of slabs 0..s-1.  Only pieces that touch a slab border can be
// joined, so every slab's map is its offset plus a short sorted list of joined labels (at most
// the number of distinct labels on its two border rows), shipped as plain arrays.
//
// The reference has no counterpart (it labels one image on one device, LabelingAlgs.cpp:989-1084);
// this is the single-image split across GPUs: one exchange of border rows, no other collective.
#include "be.h"
#include "be_api_internal.h"

#include <algorithm>
#include <cstdint>
#include <vector>

using namespace be;

namespace {

// Union-find over the border pieces, indexed in key order; the smaller index stays the root.
struct PieceSets {
    std::vector<int64_t> parent;
    explicit PieceSets(size_t n) : parent(n)
    {
        for (size_t i = 0; i < n; ++i) parent[i] = int64_t(i);
    }
    int64_t find(int64_t x)
    {
        while (parent[x] != x) {
            parent[x] = parent[parent[x]];
            x = parent[x];
        }
        return x;
    }
    void unite(int64_t a, int64_t b)
    {
        a = find(a);
        b = find(b);
        if (a < b) parent[b] = a;
        else if (b < a) parent[a] = b;
    }
};

inline uint64_t piece_key(int64_t slab, int32_t label) { return (uint64_t(slab) << 32) | uint32_t(label); }

}  // namespace

extern "C" int be_slab_merge(int32_t n_slabs, int32_t plane_rows, int32_t plane_cols, const int64_t *counts,
                             const int32_t *tops, const int32_t *bottoms, int64_t *offsets, int64_t *n_total,
                             int32_t *joined_labels, int32_t *joined_targets, int64_t *joined_start,
                             int64_t cap)
{
    if (n_slabs <= 0 || plane_rows <= 0 || plane_cols <= 0 || !counts || !tops || !bottoms || !offsets ||
        !n_total || !joined_start || cap < 0 || (cap > 0 && (!joined_labels || !joined_targets)))
        return BE_ERR_INVALID;
    const int64_t plane = int64_t(plane_rows) * plane_cols;
    for (int32_t s = 0; s < n_slabs; ++s)
        if (counts[s] < 0 || counts[s] > INT32_MAX) return BE_ERR_INVALID;

    // The pieces on the borders, in key order.
    std::vector<uint64_t> keys;
    keys.reserve(size_t(2 * plane * n_slabs / 4 + 16));
    for (int32_t s = 0; s < n_slabs; ++s) {
        for (const int32_t *row : {tops + s * plane, bottoms + s * plane}) {
            int32_t last = 0;
            for (int64_t p = 0; p < plane; ++p) {
                const int32_t l = row[p];
                if (l < 0 || l > counts[s]) return BE_ERR_INVALID;
                if (l != 0 && l != last) keys.push_back(piece_key(s, l));
                last = l;
            }
        }
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    auto index = [&](int64_t s, int32_t l) -> int64_t {
        return int64_t(std::lower_bound(keys.begin(), keys.end(), piece_key(s, l)) - keys.begin());
    };

    // Unions across every slab border.
    PieceSets sets(keys.size());
    for (int32_t s = 0; s + 1 < n_slabs; ++s) {
        const int32_t *lo = bottoms + s * plane, *hi = tops + (s + 1) * plane;
        for (int32_t r = 0; r < plane_rows; ++r) {
            for (int32_t c = 0; c < plane_cols; ++c) {
                const int32_t a = lo[int64_t(r) * plane_cols + c];
                if (!a) continue;
                int64_t ia = -1;
                for (int32_t rr = std::max(r - 1, 0); rr <= std::min(r + 1, plane_rows - 1); ++rr) {
                    for (int32_t cc = std::max(c - 1, 0); cc <= std::min(c + 1, plane_cols - 1); ++cc) {
                        const int32_t b = hi[int64_t(rr) * plane_cols + cc];
                        if (!b) continue;
                        if (ia < 0) ia = index(s, a);
                        sets.unite(ia, index(s + 1, b));
                    }
                }
            }
        }
    }

    // Joined pieces per slab (ascending labels: keys are sorted), offsets, and the joined pieces'
    // final labels.
    std::vector<int64_t> root(keys.size());
    std::vector<int64_t> start(size_t(n_slabs) + 1, 0);
    for (size_t i = 0; i < keys.size(); ++i) {
        root[i] = sets.find(int64_t(i));
        if (root[i] != int64_t(i)) ++start[size_t(keys[i] >> 32) + 1];
    }
    for (int32_t s = 0; s < n_slabs; ++s) start[s + 1] += start[s];
    if (start[n_slabs] > cap) return BE_ERR_INVALID;
    int64_t total = 0;
    for (int32_t s = 0; s < n_slabs; ++s) {
        offsets[s] = total;
        total += counts[s] - (start[s + 1] - start[s]);
    }
    if (total > INT32_MAX) return BE_ERR_INVALID;
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (size_t i = 0; i < keys.size(); ++i)
        if (root[i] != int64_t(i)) joined_labels[fill[keys[i] >> 32]++] = int32_t(keys[i] & 0xFFFFFFFFu);
    for (size_t i = 0; i < keys.size(); ++i) {
        if (root[i] == int64_t(i)) continue;
        const int64_t rs = int64_t(keys[root[i]] >> 32);
        const int32_t rl = int32_t(keys[root[i]] & 0xFFFFFFFFu);
        const int64_t below = std::lower_bound(joined_labels + start[rs], joined_labels + start[rs + 1], rl) -
                              (joined_labels + start[rs]);
        const int64_t s = int64_t(keys[i] >> 32);
        const int32_t l = int32_t(keys[i] & 0xFFFFFFFFu);
        const int64_t j = std::lower_bound(joined_labels + start[s], joined_labels + start[s + 1], l) - joined_labels;
        joined_targets[j] = int32_t(offsets[rs] + rl - below);
    }
    for (int32_t s = 0; s <= n_slabs; ++s) joined_start[s] = start[s];
    *n_total = total;
    return BE_OK;
}

namespace {

// map[l] for l = 0..count: 0 for the background, the joined piece's label for a joined label, and
// offset + l - (joined labels below l) for the others (binary search of the sorted joined list).
__global__ void k_slab_map(int32_t *map, int64_t count, int64_t offset, const int32_t *jl, const int32_t *jt, int32_t m)
{
    for (int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; l <= count; l += int64_t(gridDim.x) * blockDim.x) {
        int32_t v = 0;
        if (l > 0) {
            int32_t lo = 0, hi = m;
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (int64_t(jl[mid]) < l) lo = mid + 1;
                else hi = mid;
            }
            v = (lo < m && int64_t(jl[lo]) == l) ? jt[lo] : int32_t(offset + l - lo);
        }
        map[l] = v;
    }
}

// Labels 1..count of an n_rows x cols array (pitch in elements) through `map`, or plus `add` when
// there is no map.  Values outside 1..count are left as they are.
__device__ __forceinline__ int32_t slab_label(int32_t v, const int32_t *map, int64_t count, int32_t add)
{
    if (v <= 0 || int64_t(v) > count) return v;
    return map ? map[v] : v + add;
}

__global__ void k_slab_apply4(int4 *labels, int64_t n_rows, int32_t cols4, int64_t pitch4, const int32_t *map,
                              int64_t count, int32_t add)
{
    const int64_t n = n_rows * cols4;
    for (int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < n; u += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = u / cols4, c = u - r * cols4;
        int4 *p = labels + r * pitch4 + c;
        int4 v = *p;
        v.x = slab_label(v.x, map, count, add);
        v.y = slab_label(v.y, map, count, add);
        v.z = slab_label(v.z, map, count, add);
        v.w = slab_label(v.w, map, count, add);
        *p = v;
    }
}

__global__ void k_slab_apply(int32_t *labels, int64_t n_rows, int32_t cols, int64_t pitch, const int32_t *map,
                             int64_t count, int32_t add)
{
    const int64_t n = n_rows * cols;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = i / cols, c = i - r * cols;
        int32_t *p = labels + r * pitch + c;
        *p = slab_label(*p, map, count, add);
    }
}

unsigned slab_grid(const be_ctx *c, int64_t n)
{
    return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(c->sms) * 16)));
}

size_t al256(size_t v) { return (v + 255) / 256 * 256; }

// Grows the context's slab scratch (label map + joined lists) to hold `need` bytes.
int slab_scratch(be_ctx *c, size_t need)
{
    if (need <= c->slab_bytes) return BE_OK;
    if (c->slab_buf) cudaFree(c->slab_buf);
    c->slab_buf = nullptr;
    c->slab_bytes = 0;
    cudaError_t e = cudaMalloc(&c->slab_buf, need);
    if (e != cudaSuccess) {
        c->slab_buf = nullptr;
        return cuda_error(c, e, "be_slab scratch: cudaMalloc");
    }
    c->slab_bytes = need;
    return BE_OK;
}

size_t slab_bytes_for(int64_t count, int64_t n_joined)
{
    return al256(size_t(count + 1) * sizeof(int32_t)) + 2 * al256(size_t(n_joined) * sizeof(int32_t));
}

}  // namespace

extern "C" int be_slab_reserve(be_ctx *c, int64_t max_count, int64_t max_joined)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (max_count < 0 || max_count > INT32_MAX || max_joined < 0 || max_joined > INT32_MAX)
        return set_error(c, BE_ERR_INVALID, "be_slab_reserve: bad sizes");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaSetDevice");
    return slab_scratch(c, slab_bytes_for(max_count, max_joined));
}

extern "C" int be_slab_relabel(be_ctx *c, int32_t *labels, int64_t n_rows, int32_t cols, int64_t pitch,
                               int64_t count, int64_t offset, const int32_t *joined_labels,
                               const int32_t *joined_targets, int32_t n_joined, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!labels || n_rows <= 0 || cols <= 0 || pitch < cols || count < 0 || count > INT32_MAX || offset < 0 ||
        offset + count > INT32_MAX || n_joined < 0 || (n_joined > 0 && (!joined_labels || !joined_targets)))
        return set_error(c, BE_ERR_INVALID, "be_slab_relabel: bad arguments");
    if (n_joined == 0 && offset == 0) return BE_OK;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaSetDevice");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int32_t *map = nullptr;
    if (n_joined > 0) {
        const size_t o_jl = al256(size_t(count + 1) * sizeof(int32_t));
        const size_t o_jt = o_jl + al256(size_t(n_joined) * sizeof(int32_t));
        const int rc = slab_scratch(c, slab_bytes_for(count, n_joined));
        if (rc) return rc;
        char *base = static_cast<char *>(c->slab_buf);
        int32_t *d_map = reinterpret_cast<int32_t *>(base);
        int32_t *d_jl = reinterpret_cast<int32_t *>(base + o_jl), *d_jt = reinterpret_cast<int32_t *>(base + o_jt);
        e = cudaMemcpyAsync(d_jl, joined_labels, size_t(n_joined) * sizeof(int32_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_jt, joined_targets, size_t(n_joined) * sizeof(int32_t), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_error(c, e, "be_slab_relabel: upload");
        k_slab_map<<<slab_grid(c, count + 1), 256, 0, s>>>(d_map, count, offset, d_jl, d_jt, n_joined);
        map = d_map;
    }
    const bool vec = cols % 4 == 0 && pitch % 4 == 0 && (reinterpret_cast<uintptr_t>(labels) & 15) == 0;
    if (vec)
        k_slab_apply4<<<slab_grid(c, n_rows * (cols / 4)), 256, 0, s>>>(reinterpret_cast<int4 *>(labels), n_rows,
                                                                        cols / 4, pitch / 4, map, count,
                                                                        int32_t(offset));
    else
        k_slab_apply<<<slab_grid(c, n_rows * cols), 256, 0, s>>>(labels, n_rows, cols, pitch, map, count,
                                                                 int32_t(offset));
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(c, e, "be_slab_relabel launch");
    return BE_OK;
}

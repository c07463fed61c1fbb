// be_iter.cu -- the paper's iterative Block-Equivalence merge ("plain form", BE_ALGO_ITER).
//
// Same algorithm as the reference's LBEQ2_* / BLEQ3D_* kernels (LabelingAlgs.cl:176-319,
// 805-979) driven by LabelSPixels (LabelingAlgs.cpp:1014-1039 / 1467-1492):
//   init     per block: foreground mask, label = first-pixel key + 1 (0 = empty block)
//   conn     per block: bit d set when the block touches its neighbour d (8 / 26 neighbours)
//   loop     Scan: m = min label of connected neighbours; if m < label, lower the label's root
//            entry to m (atomicMin here; the reference's plain store is racy) and flag a change.
//            Analyze: chase each label to its root (bounded; path compression).
//   final    canonical rank of each root key, then the per-pixel write.
// Differences from the reference, by design:
//   * labels are first-pixel keys instead of block indices, so roots end at each component's
//     first pixel in raster order and the ranks are canonical;
//   * the loop runs inside one CUDA graph: a conditional WHILE node repeats {Scan, Analyze,
//     check} until a device-side flag says nothing changed -- no host round trip per iteration
//     (the reference does a blocking flag read each time, LabelingAlgs.cpp:1034);
//   * an iteration cap ends the loop with BE_ERR_NO_CONVERGENCE instead of spinning forever.
// Keys use power-of-two row lengths so a key decodes to its block with shifts:
// 2D key = (y << sx) | x; 3D key = (((X << s1) | Y) << s2) | Z.
#include "be.h"
#include "be_api_internal.h"
#include "be_kernels.h"

#include <algorithm>
#include <cstring>

namespace be {

namespace {

constexpr int kIterCap = 4096;        // Scan/Analyze rounds before BE_ERR_NO_CONVERGENCE
constexpr int kChaseCap = 1 << 22;    // steps of one root chase before the error flag is set
constexpr int NT = 256;

struct It2 {
    const uint8_t *in;
    int64_t pitch;
    int32_t *out;
    int64_t opitch;
    int rows, cols, bw, bh, sx, thr;
    uint32_t *lab;     // per block: root key + 1, 0 = empty
    uint8_t *mk;       // per block: mask
    uint8_t *conn;     // per block: 8 neighbour bits (reference order, LabelingAlgs.cl:163-167)
    uint32_t *rbits;   // root bitmap over keys
    uint32_t *ctl;     // [0] changed, [1] iteration, [2] error
    Work w;            // segment machinery over root-bitmap words
};

struct It3 {
    const uint8_t *in;
    int32_t *out;
    int d0, d1, d2, b0, b1, b2, s1, s2, thr;
    uint32_t *lab;
    uint8_t *mk;
    uint32_t *conn;    // 26 neighbour bits, bit (dx+1) + 3(dy+1) + 9(dz+1) (LabelingAlgs.cl:762-768)
    uint32_t *rbits;
    uint32_t *ctl;
    Work w;
};

__device__ __forceinline__ uint32_t sel2(int dx, int dy)
{
    const uint32_t sx = dx < 0 ? 0x5u : dx > 0 ? 0xAu : 0xFu;   // mask bit = 2*row + col
    const uint32_t sy = dy < 0 ? 0x3u : dy > 0 ? 0xCu : 0xFu;
    return sx & sy;
}

__device__ __forceinline__ uint32_t sel3(int dx, int dy, int dz)
{
    const uint32_t a = dx < 0 ? 0x0Fu : dx > 0 ? 0xF0u : 0xFFu;
    const uint32_t b = dy < 0 ? 0x33u : dy > 0 ? 0xCCu : 0xFFu;
    const uint32_t c = dz < 0 ? 0x55u : dz > 0 ? 0xAAu : 0xFFu;
    return a & b & c;
}

// ---- 2D -------------------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) it_init_2d(It2 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.bw) * g.bh) return;
    const int by = int(b / g.bw), bx = int(b - int64_t(by) * g.bw);
    const int y = 2 * by, x = 2 * bx;
    const uint8_t *p = g.in + int64_t(y) * g.pitch + x;
    const bool xr = x + 1 < g.cols, yb = y + 1 < g.rows;
    uint32_t m = (p[0] > g.thr) | (xr && p[1] > g.thr) << 1;
    if (yb) m |= (p[g.pitch] > g.thr) << 2 | (xr && p[g.pitch + 1] > g.thr) << 3;
    g.mk[b] = uint8_t(m);
    uint32_t lab = 0;
    if (m) {
        const int fy = (m & 3u) ? 0 : 1;
        const int fx = (m & 3u) ? ((m & 1u) ? 0 : 1) : ((m & 4u) ? 0 : 1);
        lab = ((uint32_t(y + fy) << g.sx) | uint32_t(x + fx)) + 1u;
    }
    g.lab[b] = lab;
}

__global__ void __launch_bounds__(NT) it_conn_2d(It2 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.bw) * g.bh) return;
    const int by = int(b / g.bw), bx = int(b - int64_t(by) * g.bw);
    const uint32_t m = g.mk[b];
    uint32_t c = 0;
    if (m) {
        constexpr int DX[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
        constexpr int DY[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int nx = bx + DX[k], ny = by + DY[k];
            if (nx < 0 || ny < 0 || nx >= g.bw || ny >= g.bh) continue;
            const uint32_t mn = g.mk[int64_t(ny) * g.bw + nx];
            if ((m & sel2(DX[k], DY[k])) && (mn & sel2(-DX[k], -DY[k]))) c |= 1u << k;
        }
    }
    g.conn[b] = uint8_t(c);
}

__device__ __forceinline__ int64_t key_block_2d(const It2 &g, uint32_t key)
{
    const uint32_t y = key >> g.sx, x = key & ((1u << g.sx) - 1u);
    return int64_t(y >> 1) * g.bw + (x >> 1);
}

__global__ void __launch_bounds__(NT) it_scan_2d(It2 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.bw) * g.bh) return;
    const uint32_t label = g.lab[b];
    if (!label) return;
    const uint32_t c = g.conn[b];
    if (!c) return;
    const int by = int(b / g.bw), bx = int(b - int64_t(by) * g.bw);
    constexpr int DX[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
    constexpr int DY[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    uint32_t m = 0xFFFFFFFFu;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if (c & (1u << k)) m = min(m, g.lab[int64_t(by + DY[k]) * g.bw + bx + DX[k]]);
    if (m < label) {
        atomicMin(&g.lab[key_block_2d(g, label - 1)], m);
        g.ctl[0] = 1;
    }
}

__global__ void __launch_bounds__(NT) it_analyze_2d(It2 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.bw) * g.bh) return;
    uint32_t label = g.lab[b];
    if (!label) return;
    for (int step = 0;; ++step) {
        const uint32_t nxt = g.lab[key_block_2d(g, label - 1)];
        if (nxt == label) break;
        if (step == kChaseCap) { g.ctl[2] = 1; break; }
        label = nxt;
    }
    g.lab[b] = label;
}

__global__ void __launch_bounds__(NT) it_mark_2d(It2 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.bw) * g.bh) return;
    const uint32_t label = g.lab[b];
    if (!label || key_block_2d(g, label - 1) != b) return;
    const uint32_t k = label - 1;
    atomicOr(&g.rbits[k >> 5], 1u << (k & 31));
}

__global__ void __launch_bounds__(NT) it_final_2d(It2 g)
{
    const int64_t u = int64_t(blockIdx.x) * NT + threadIdx.x;   // one unit = 2 pixels (1 block row)
    const int64_t per_row = g.bw;
    if (u >= per_row * g.rows) return;
    const int y = int(u / per_row), bx = int(u - int64_t(y) * per_row);
    const int64_t b = int64_t(y >> 1) * g.bw + bx;
    const uint32_t m = g.mk[b];
    uint32_t l = 0;
    if (m) {
        const uint32_t k = g.lab[b] - 1;
        l = 1u + g.w.segpref[k >> 5] + __popc(g.rbits[k >> 5] & ((1u << (k & 31)) - 1u));
    }
    const int h = (y & 1) * 2;
    int32_t *dst = g.out + int64_t(y) * g.opitch + 2 * bx;
    dst[0] = ((m >> h) & 1u) ? int(l) : 0;
    if (2 * bx + 1 < g.cols) dst[1] = ((m >> (h + 1)) & 1u) ? int(l) : 0;
}

// ---- 3D -------------------------------------------------------------------------------------
__device__ __forceinline__ int64_t key_block_3d(const It3 &g, uint32_t key)
{
    const uint32_t Z = key & ((1u << g.s2) - 1u);
    const uint32_t Y = (key >> g.s2) & ((1u << g.s1) - 1u);
    const uint32_t X = key >> (g.s1 + g.s2);
    return (int64_t(X >> 1) * g.b1 + (Y >> 1)) * g.b2 + (Z >> 1);
}

__global__ void __launch_bounds__(NT) it_init_3d(It3 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    const int64_t nb = int64_t(g.b0) * g.b1 * g.b2;
    if (b >= nb) return;
    const int bz = int(b % g.b2), by = int((b / g.b2) % g.b1), bx = int(b / (int64_t(g.b2) * g.b1));
    uint32_t m = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const int X = 2 * bx + (v >> 2), Y = 2 * by + ((v >> 1) & 1), Z = 2 * bz + (v & 1);
        if (X < g.d0 && Y < g.d1 && Z < g.d2 && g.in[(int64_t(X) * g.d1 + Y) * g.d2 + Z] > g.thr)
            m |= 1u << v;
    }
    g.mk[b] = uint8_t(m);
    uint32_t lab = 0;
    if (m) {
        const int v = __ffs(m) - 1;
        const uint32_t X = 2 * bx + (v >> 2), Y = 2 * by + ((v >> 1) & 1), Z = 2 * bz + (v & 1);
        lab = ((((X << g.s1) | Y) << g.s2) | Z) + 1u;
    }
    g.lab[b] = lab;
}

__global__ void __launch_bounds__(NT) it_conn_3d(It3 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    const int64_t nb = int64_t(g.b0) * g.b1 * g.b2;
    if (b >= nb) return;
    const int bz = int(b % g.b2), by = int((b / g.b2) % g.b1), bx = int(b / (int64_t(g.b2) * g.b1));
    const uint32_t m = g.mk[b];
    uint32_t c = 0;
    if (m) {
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dx && !dy && !dz) continue;
                    const int nx = bx + dx, ny = by + dy, nz = bz + dz;
                    if (nx < 0 || ny < 0 || nz < 0 || nx >= g.b0 || ny >= g.b1 || nz >= g.b2) continue;
                    const uint32_t mn = g.mk[(int64_t(nx) * g.b1 + ny) * g.b2 + nz];
                    if ((m & sel3(dx, dy, dz)) && (mn & sel3(-dx, -dy, -dz)))
                        c |= 1u << ((dx + 1) + 3 * (dy + 1) + 9 * (dz + 1));
                }
    }
    g.conn[b] = c;
}

__global__ void __launch_bounds__(NT) it_scan_3d(It3 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    const int64_t nb = int64_t(g.b0) * g.b1 * g.b2;
    if (b >= nb) return;
    const uint32_t label = g.lab[b];
    if (!label) return;
    uint32_t c = g.conn[b];
    if (!c) return;
    uint32_t m = 0xFFFFFFFFu;
    while (c) {
        const int k = __ffs(c) - 1;
        c &= c - 1;
        const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
        m = min(m, g.lab[b + (int64_t(dx) * g.b1 + dy) * g.b2 + dz]);
    }
    if (m < label) {
        atomicMin(&g.lab[key_block_3d(g, label - 1)], m);
        g.ctl[0] = 1;
    }
}

__global__ void __launch_bounds__(NT) it_analyze_3d(It3 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.b0) * g.b1 * g.b2) return;
    uint32_t label = g.lab[b];
    if (!label) return;
    for (int step = 0;; ++step) {
        const uint32_t nxt = g.lab[key_block_3d(g, label - 1)];
        if (nxt == label) break;
        if (step == kChaseCap) { g.ctl[2] = 1; break; }
        label = nxt;
    }
    g.lab[b] = label;
}

__global__ void __launch_bounds__(NT) it_mark_3d(It3 g)
{
    const int64_t b = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (b >= int64_t(g.b0) * g.b1 * g.b2) return;
    const uint32_t label = g.lab[b];
    if (!label || key_block_3d(g, label - 1) != b) return;
    const uint32_t k = label - 1;
    atomicOr(&g.rbits[k >> 5], 1u << (k & 31));
}

__global__ void __launch_bounds__(NT) it_final_3d(It3 g)
{
    const int64_t v = int64_t(blockIdx.x) * NT + threadIdx.x;
    const int64_t n = int64_t(g.d0) * g.d1 * g.d2;
    if (v >= n) return;
    const int Z = int(v % g.d2), Y = int((v / g.d2) % g.d1), X = int(v / (int64_t(g.d2) * g.d1));
    const int64_t b = (int64_t(X >> 1) * g.b1 + (Y >> 1)) * g.b2 + (Z >> 1);
    const uint32_t m = g.mk[b];
    const int bit = 4 * (X & 1) + 2 * (Y & 1) + (Z & 1);
    int32_t l = 0;
    if ((m >> bit) & 1u) {
        const uint32_t k = g.lab[b] - 1;
        l = int32_t(1u + g.w.segpref[k >> 5] + __popc(g.rbits[k >> 5] & ((1u << (k & 31)) - 1u)));
    }
    g.out[v] = l;
}

// ---- shared by both ---------------------------------------------------------------------------
__global__ void it_cond(cudaGraphConditionalHandle h, uint32_t *ctl)
{
    const uint32_t changed = ctl[0];
    ctl[0] = 0;
    const uint32_t it = ++ctl[1];
    unsigned go = changed ? 1u : 0u;
    if (go && it >= uint32_t(kIterCap)) {
        ctl[2] = 1;
        go = 0;
    }
    if (ctl[2]) go = 0;
    cudaGraphSetConditional(h, go);
}

__global__ void __launch_bounds__(NT) it_count(const uint32_t *rbits, uint8_t *cnt, int64_t n)
{
    const int64_t i = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (i < n) cnt[i] = uint8_t(__popc(rbits[i]));
}

__global__ void it_ncomp(Work w, const uint32_t *ctl, uint32_t *err_out)
{
    w.ncomp[0] = int64_t(w.segpref[w.n_segs]);
    *err_out = ctl[2];
}

// ---- pixel-level label equivalence (-a lbeq -g) ------------------------------------------------
// The reference's DistrInit/Scan/Analize (LabelingAlgs.cl:31-130) and LBEQ3D_* (:635-734):
// every foreground pixel starts with its own label and the Scan / Analyze loop of the block form
// runs on pixels.  2D: 4 neighbours (COH_4 and the reference's default) or 8 (COH_8); 3D: 26.
// Labels are first-pixel keys as in the block form, so the output is canonical; the reference's
// own quirk (a foreground pixel at (0, 0) keeps label 0, LabelingAlgs.cl:37, 48-50) is not
// reproduced.
struct Lq2 {
    const uint8_t *in;
    int64_t pitch;
    int32_t *out;
    int64_t opitch;
    int rows, cols, sx, thr, conn8;
    uint32_t *lab;
    uint32_t *rbits;
    uint32_t *ctl;
    Work w;
};

struct Lq3 {
    const uint8_t *in;
    int32_t *out;
    int d0, d1, d2, s1, s2, thr;
    uint32_t *lab;
    uint32_t *rbits;
    uint32_t *ctl;
    Work w;
};

__device__ __forceinline__ int64_t lq_pix2(const Lq2 &g, uint32_t key)
{
    return int64_t(key >> g.sx) * g.cols + (key & ((1u << g.sx) - 1u));
}

__global__ void __launch_bounds__(NT) lq_init_2d(Lq2 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.rows) * g.cols) return;
    const int y = int(p / g.cols), x = int(p - int64_t(y) * g.cols);
    g.lab[p] = g.in[int64_t(y) * g.pitch + x] > g.thr ? ((uint32_t(y) << g.sx) | uint32_t(x)) + 1u : 0u;
}

__global__ void __launch_bounds__(NT) lq_scan_2d(Lq2 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.rows) * g.cols) return;
    const uint32_t label = g.lab[p];
    if (!label) return;
    const int y = int(p / g.cols), x = int(p - int64_t(y) * g.cols);
    uint32_t m = 0xFFFFFFFFu;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            if ((!dx && !dy) || (!g.conn8 && dx && dy)) continue;
            const int ny = y + dy, nx = x + dx;
            if (ny < 0 || nx < 0 || ny >= g.rows || nx >= g.cols) continue;
            const uint32_t v = g.lab[int64_t(ny) * g.cols + nx];
            if (v && v < m) m = v;
        }
    if (m < label) {
        atomicMin(&g.lab[lq_pix2(g, label - 1)], m);
        g.ctl[0] = 1;
    }
}

__global__ void __launch_bounds__(NT) lq_analyze_2d(Lq2 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.rows) * g.cols) return;
    uint32_t label = g.lab[p];
    if (!label) return;
    for (int step = 0;; ++step) {
        const uint32_t nxt = g.lab[lq_pix2(g, label - 1)];
        if (nxt == label) break;
        if (step == kChaseCap) { g.ctl[2] = 1; break; }
        label = nxt;
    }
    g.lab[p] = label;
}

__global__ void __launch_bounds__(NT) lq_mark_2d(Lq2 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.rows) * g.cols) return;
    const uint32_t label = g.lab[p];
    if (!label || lq_pix2(g, label - 1) != p) return;
    const uint32_t k = label - 1;
    atomicOr(&g.rbits[k >> 5], 1u << (k & 31));
}

__global__ void __launch_bounds__(NT) lq_final_2d(Lq2 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.rows) * g.cols) return;
    const int y = int(p / g.cols), x = int(p - int64_t(y) * g.cols);
    const uint32_t label = g.lab[p];
    int32_t l = 0;
    if (label) {
        const uint32_t k = label - 1;
        l = int32_t(1u + g.w.segpref[k >> 5] + __popc(g.rbits[k >> 5] & ((1u << (k & 31)) - 1u)));
    }
    g.out[int64_t(y) * g.opitch + x] = l;
}

__device__ __forceinline__ int64_t lq_pix3(const Lq3 &g, uint32_t key)
{
    const uint32_t Z = key & ((1u << g.s2) - 1u);
    const uint32_t Y = (key >> g.s2) & ((1u << g.s1) - 1u);
    const uint32_t X = key >> (g.s1 + g.s2);
    return (int64_t(X) * g.d1 + Y) * g.d2 + Z;
}

__global__ void __launch_bounds__(NT) lq_init_3d(Lq3 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.d0) * g.d1 * g.d2) return;
    const uint32_t Z = uint32_t(p % g.d2), Y = uint32_t((p / g.d2) % g.d1), X = uint32_t(p / (int64_t(g.d2) * g.d1));
    g.lab[p] = g.in[p] > g.thr ? ((((X << g.s1) | Y) << g.s2) | Z) + 1u : 0u;
}

__global__ void __launch_bounds__(NT) lq_scan_3d(Lq3 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.d0) * g.d1 * g.d2) return;
    const uint32_t label = g.lab[p];
    if (!label) return;
    const int Z = int(p % g.d2), Y = int((p / g.d2) % g.d1), X = int(p / (int64_t(g.d2) * g.d1));
    uint32_t m = 0xFFFFFFFFu;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                const int nx = X + dx, ny = Y + dy, nz = Z + dz;
                if (nx < 0 || ny < 0 || nz < 0 || nx >= g.d0 || ny >= g.d1 || nz >= g.d2) continue;
                const uint32_t v = g.lab[(int64_t(nx) * g.d1 + ny) * g.d2 + nz];
                if (v && v < m) m = v;
            }
    if (m < label) {
        atomicMin(&g.lab[lq_pix3(g, label - 1)], m);
        g.ctl[0] = 1;
    }
}

__global__ void __launch_bounds__(NT) lq_analyze_3d(Lq3 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.d0) * g.d1 * g.d2) return;
    uint32_t label = g.lab[p];
    if (!label) return;
    for (int step = 0;; ++step) {
        const uint32_t nxt = g.lab[lq_pix3(g, label - 1)];
        if (nxt == label) break;
        if (step == kChaseCap) { g.ctl[2] = 1; break; }
        label = nxt;
    }
    g.lab[p] = label;
}

__global__ void __launch_bounds__(NT) lq_mark_3d(Lq3 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.d0) * g.d1 * g.d2) return;
    const uint32_t label = g.lab[p];
    if (!label || lq_pix3(g, label - 1) != p) return;
    const uint32_t k = label - 1;
    atomicOr(&g.rbits[k >> 5], 1u << (k & 31));
}

__global__ void __launch_bounds__(NT) lq_final_3d(Lq3 g)
{
    const int64_t p = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (p >= int64_t(g.d0) * g.d1 * g.d2) return;
    const uint32_t label = g.lab[p];
    int32_t l = 0;
    if (label) {
        const uint32_t k = label - 1;
        l = int32_t(1u + g.w.segpref[k >> 5] + __popc(g.rbits[k >> 5] & ((1u << (k & 31)) - 1u)));
    }
    g.out[p] = l;
}

// ---- run equivalence (-a runeq -g) -------------------------------------------------------------
// The reference's TOCLRunEquivLabeling (LabelingAlgs.cpp:1090-1268, kernels RE* in
// LabelingAlgs.cl:325-616): the nodes are the horizontal runs of each row; every run is given the
// range of runs it overlaps in the row above and below; the Scan / Analyze loop then lowers each
// run's root label to the smallest label among its neighbours and chases labels to their roots
// until nothing changes; the final pass writes each run's label over its pixels.  The reference's
// runs overlap by column only (4-connectivity); conn8 also joins runs that touch diagonally.
// Differences, by design:
//   * one warp per row finds the row's runs with ballot-free bit operations on 32-pixel words
//     (foreground, run-start and run-end words, starts counted by a warp prefix sum), where the
//     reference walks each row pixel by pixel in one thread (REFindRunsKernel);
//   * a run's neighbour ranges come from the start-bit words in O(1) (count of run starts up to a
//     column), not from a linear walk of the neighbouring row (FindNeibRuns);
//   * the label is the run's index + 1 in raster order (row, then column), so roots end at each
//     component's first run and its first pixel, and the output is canonical (first-pixel order);
//   * the loop runs inside the iterative form's CUDA graph (device-side WHILE, iteration cap).
struct Re2 {
    const uint8_t *in;
    int64_t pitch;
    int32_t *out;
    int64_t opitch;
    int rows, cols, sx, thr, conn8;
    int words;          // 32-pixel words per row
    int rmax;           // run capacity per row: (cols + 1) / 2
    uint32_t *fgb;      // [rows][words] foreground bits
    uint32_t *stb;      // [rows][words] run-start bits
    uint32_t *spre;     // [rows][words] run starts of the row before the word
    uint32_t *nrun;     // [rows] runs of the row
    int32_t *rl, *rr;   // [rows][rmax] first and last column of each run
    uint32_t *lab;      // [rows][rmax] label: index + 1 of the run's current root run
    uint4 *nb;          // [rows][rmax] overlapped runs (indices in their row): above first / last,
                        //              below first / last (first > last: none)
    uint32_t *rbits;    // root bitmap over first-pixel keys (y << sx) | x
    uint32_t *ctl;
    Work w;
};

// Foreground bits of 32 pixels starting at column x0 of row y (pixels past the row are 0).
__device__ __forceinline__ uint32_t re_word(const Re2 &g, int y, int x0)
{
    const uint8_t *p = g.in + int64_t(y) * g.pitch + x0;
    uint32_t m = 0;
    if (x0 + 32 <= g.cols && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
        const uint4 a = __ldg(reinterpret_cast<const uint4 *>(p)), b = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
        const uint32_t v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int k = 0; k < 4; ++k) m |= uint32_t(((v[i] >> (8 * k)) & 0xFFu) > uint32_t(g.thr)) << (4 * i + k);
    } else {
        const int n = min(32, g.cols - x0);
        for (int k = 0; k < n; ++k) m |= uint32_t(p[k] > g.thr) << k;
    }
    return m;
}

// One warp per row: the row's foreground / run-start words, the starts before each word, and the
// runs' extents and initial labels.
__global__ void __launch_bounds__(NT) re_rows(Re2 g)
{
    const int64_t gw = (int64_t(blockIdx.x) * NT + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= g.rows) return;   // whole warps leave together
    const int y = int(gw);
    uint32_t *fgb = g.fgb + int64_t(y) * g.words, *stb = g.stb + int64_t(y) * g.words;
    uint32_t *spre = g.spre + int64_t(y) * g.words;
    const int64_t rbase = int64_t(y) * g.rmax;
    uint32_t carry = 0, offset = 0;   // last pixel of the previous chunk, starts before the chunk
    for (int base = 0; base < g.words; base += 32) {
        const int wd = base + lane;
        const uint32_t f = wd < g.words ? re_word(g, y, 32 * wd) : 0u;
        const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, f, 1);
        const uint32_t prev = lane ? (up >> 31) : carry;
        const uint32_t st = f & ~((f << 1) | prev);
        uint32_t nxt = __shfl_down_sync(0xFFFFFFFFu, f, 1) & 1u;
        if (lane == 31) nxt = (32 * (wd + 1) < g.cols) ? uint32_t(g.in[int64_t(y) * g.pitch + 32 * (wd + 1)] > g.thr) : 0u;
        const uint32_t en = f & ~((f >> 1) | (nxt << 31));
        // exclusive prefix of the starts over the warp
        const uint32_t c = __popc(st);
        uint32_t inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (lane >= o) inc += v;
        }
        const uint32_t pre = offset + inc - c;
        if (wd < g.words) {
            fgb[wd] = f;
            stb[wd] = st;
            spre[wd] = pre;
            uint32_t b = st;
            for (uint32_t k = pre; b; ++k) {
                const int bit = __ffs(b) - 1;
                b &= b - 1;
                g.rl[rbase + k] = 32 * wd + bit;
                g.lab[rbase + k] = uint32_t(rbase + k) + 1u;
            }
            // a run ends in this word: it is the last run started at or before that bit
            b = en;
            while (b) {
                const int bit = __ffs(b) - 1;
                b &= b - 1;
                const uint32_t k = pre + __popc(st & (0xFFFFFFFFu >> (31 - bit))) - 1u;
                g.rr[rbase + k] = 32 * wd + bit;
            }
        }
        offset = __shfl_sync(0xFFFFFFFFu, pre + c, 31);
        carry = __shfl_sync(0xFFFFFFFFu, f, 31) >> 31;
    }
    if (lane == 0) g.nrun[y] = offset;
}

// Runs of row y started at or before column x (x may be -1: none).
__device__ __forceinline__ uint32_t re_starts_upto(const Re2 &g, int y, int x)
{
    if (x < 0) return 0u;
    const int wd = x >> 5;
    const int64_t i = int64_t(y) * g.words + wd;
    return g.spre[i] + __popc(g.stb[i] & (0xFFFFFFFFu >> (31 - (x & 31))));
}

// Range of runs of row y that overlap columns [a, b] (clipped to the row): first > last when none.
__device__ __forceinline__ uint2 re_range(const Re2 &g, int y, int a, int b)
{
    a = max(a, 0);
    b = min(b, g.cols - 1);
    if (a > b) return make_uint2(1u, 0u);
    const bool fa = (g.fgb[int64_t(y) * g.words + (a >> 5)] >> (a & 31)) & 1u;
    const uint32_t first = re_starts_upto(g, y, a) - (fa ? 1u : 0u);
    const uint32_t last = re_starts_upto(g, y, b);   // one past the last
    return last > first ? make_uint2(first, last - 1u) : make_uint2(1u, 0u);
}

__global__ void __launch_bounds__(NT) re_nbr(Re2 g)
{
    const int64_t i = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (i >= int64_t(g.rows) * g.rmax) return;
    const int y = int(i / g.rmax), k = int(i - int64_t(y) * g.rmax);
    if (uint32_t(k) >= g.nrun[y]) return;
    const int a = g.rl[i] - g.conn8, b = g.rr[i] + g.conn8;
    const uint2 up = y > 0 ? re_range(g, y - 1, a, b) : make_uint2(1u, 0u);
    const uint2 dn = y + 1 < g.rows ? re_range(g, y + 1, a, b) : make_uint2(1u, 0u);
    g.nb[i] = make_uint4(up.x, up.y, dn.x, dn.y);
}

// Scan: the smallest label among the overlapped runs lowers this run's root (REScanKernel,
// LabelingAlgs.cl:555-577; atomicMin where the reference stores).
__global__ void __launch_bounds__(NT) re_scan(Re2 g)
{
    const int64_t i = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (i >= int64_t(g.rows) * g.rmax) return;
    const int y = int(i / g.rmax), k = int(i - int64_t(y) * g.rmax);
    if (uint32_t(k) >= g.nrun[y]) return;
    const uint32_t label = g.lab[i];
    const uint4 r = g.nb[i];
    uint32_t m = label;
    for (uint32_t j = r.x; j <= r.y && r.x <= r.y; ++j) m = min(m, g.lab[int64_t(y - 1) * g.rmax + j]);
    for (uint32_t j = r.z; j <= r.w && r.z <= r.w; ++j) m = min(m, g.lab[int64_t(y + 1) * g.rmax + j]);
    if (m < label) {
        atomicMin(&g.lab[label - 1], m);
        g.ctl[0] = 1u;
    }
}

// Analyze: every run's label chased to its root (REAnalizeKernel, LabelingAlgs.cl:581-601).
__global__ void __launch_bounds__(NT) re_analyze(Re2 g)
{
    const int64_t i = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (i >= int64_t(g.rows) * g.rmax) return;
    const int y = int(i / g.rmax), k = int(i - int64_t(y) * g.rmax);
    if (uint32_t(k) >= g.nrun[y]) return;
    uint32_t l = g.lab[i], c = g.lab[l - 1];
    int steps = 0;
    while (c != l) {
        if (++steps > kChaseCap) {
            g.ctl[2] = 1u;
            return;
        }
        l = c;
        c = g.lab[l - 1];
    }
    g.lab[i] = l;
}

// Roots mark their first pixel in the root bitmap.
__global__ void __launch_bounds__(NT) re_mark(Re2 g)
{
    const int64_t i = int64_t(blockIdx.x) * NT + threadIdx.x;
    if (i >= int64_t(g.rows) * g.rmax) return;
    const int y = int(i / g.rmax), k = int(i - int64_t(y) * g.rmax);
    if (uint32_t(k) >= g.nrun[y] || g.lab[i] != uint32_t(i) + 1u) return;
    const uint32_t key = (uint32_t(y) << g.sx) | uint32_t(g.rl[i]);
    atomicOr(&g.rbits[key >> 5], 1u << (key & 31));
}

// Final write (RELabelKernel, LabelingAlgs.cl:605-620): four pixels per thread; a foreground
// pixel's run is the last run started at or before it, its label the canonical rank of the
// run's root's first pixel.
__global__ void __launch_bounds__(NT) re_final(Re2 g)
{
    const int64_t u = int64_t(blockIdx.x) * NT + threadIdx.x;
    const int units = (g.cols + 3) >> 2;
    if (u >= int64_t(g.rows) * units) return;
    const int y = int(u / units), x0 = 4 * int(u - int64_t(y) * units);
    const uint32_t f = g.fgb[int64_t(y) * g.words + (x0 >> 5)] >> (x0 & 31);
    int v[4] = {0, 0, 0, 0};
    uint32_t run = 0xFFFFFFFFu, lbl = 0;
    for (int q = 0; q < 4 && x0 + q < g.cols; ++q) {
        if (!((f >> q) & 1u)) continue;
        const uint32_t r = re_starts_upto(g, y, x0 + q) - 1u;
        if (r != run) {
            run = r;
            const uint32_t root = g.lab[int64_t(y) * g.rmax + r] - 1u;
            const uint32_t ry = root / uint32_t(g.rmax);
            const uint32_t key = (ry << g.sx) | uint32_t(g.rl[root]);
            lbl = 1u + g.w.segpref[key >> 5] + __popc(g.rbits[key >> 5] & ((1u << (key & 31)) - 1u));
        }
        v[q] = int(lbl);
    }
    int32_t *dst = g.out + int64_t(y) * g.opitch + x0;
    if (x0 + 4 <= g.cols && ((reinterpret_cast<uintptr_t>(dst) & 15) == 0)) {
        *reinterpret_cast<int4 *>(dst) = make_int4(v[0], v[1], v[2], v[3]);
    } else {
        for (int q = 0; q < 4 && x0 + q < g.cols; ++q) dst[q] = v[q];
    }
}

unsigned nblk(int64_t n) { return unsigned((n + NT - 1) / NT); }

int ceil_log2(int v)
{
    int s = 0;
    while ((1 << s) < v) ++s;
    return s;
}

// Adds a kernel node with the given arguments to `graph` after `dep` (may be null).
template <class... A>
cudaError_t add_kernel(cudaGraph_t graph, cudaGraphNode_t *node, cudaGraphNode_t dep, void (*fn)(A...),
                       unsigned grid, unsigned block, A... args)
{
    void *argv[] = {static_cast<void *>(&args)...};
    cudaKernelNodeParams p = {};
    p.func = reinterpret_cast<void *>(fn);
    p.gridDim = dim3(std::max(grid, 1u));
    p.blockDim = dim3(block);
    p.sharedMemBytes = 0;
    p.kernelParams = argv;
    return cudaGraphAddKernelNode(node, graph, dep ? &dep : nullptr, dep ? 1 : 0, &p);
}

// Scratch of the iterative form: block labels, masks, connectivity, root bitmap and the segment
// workspace (over bitmap words), carved from the context's iteration buffer.
int iter_scratch(be_ctx *c, int64_t nblocks, size_t conn_bytes, int64_t nwords, char **lab, char **mk,
                 char **conn, char **rbits, char **ctl, size_t extra_bytes = 0, char **extra = nullptr)
{
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    const size_t need = al(nblocks * 4) + al(nblocks) + al(nblocks * conn_bytes) + al(nwords * 4) + 256 +
                        al(extra_bytes);
    if (need > c->iter_bytes) {
        if (c->iter_base) cudaFree(c->iter_base);
        c->iter_base = nullptr;
        c->iter_bytes = 0;
        cudaError_t e = cudaMalloc(&c->iter_base, need);
        if (e != cudaSuccess) return cuda_error(c, e, "cudaMalloc(iteration scratch)");
        c->iter_bytes = need;
    }
    char *p = static_cast<char *>(c->iter_base);
    *lab = p; p += al(nblocks * 4);
    *mk = p; p += al(nblocks);
    *conn = p; p += al(nblocks * conn_bytes);
    *rbits = p; p += al(nwords * 4);
    *ctl = p; p += 256;
    if (extra) *extra = p;
    if (!c->iter_err) {
        cudaError_t e = cudaMallocHost(&c->iter_err, 16);
        if (e != cudaSuccess) return cuda_error(c, e, "cudaMallocHost(iteration flag)");
    }
    return BE_OK;
}

// The arguments that only the init and final kernels read (the image buffers and threshold),
// blanked for the graph cache's key.
void blank_io(It2 &g) { g.in = nullptr; g.out = nullptr; g.pitch = g.opitch = 0; g.thr = 0; }
void blank_io(It3 &g) { g.in = nullptr; g.out = nullptr; g.thr = 0; }
void blank_io(Lq2 &g) { g.in = nullptr; g.out = nullptr; g.pitch = g.opitch = 0; g.thr = 0; }
void blank_io(Lq3 &g) { g.in = nullptr; g.out = nullptr; g.thr = 0; }
void blank_io(Re2 &g) { g.in = nullptr; g.out = nullptr; g.pitch = g.opitch = 0; g.thr = 0; }

template <class G>
cudaError_t set_kernel_args(cudaGraphExec_t exec, cudaGraphNode_t node, void *fn, unsigned grid, G &g)
{
    void *argv[] = {static_cast<void *>(&g)};
    cudaKernelNodeParams p = {};
    p.func = fn;
    p.gridDim = dim3(std::max(grid, 1u));
    p.blockDim = dim3(NT);
    p.sharedMemBytes = 0;
    p.kernelParams = argv;
    return cudaGraphExecKernelNodeSetParams(exec, node, &p);
}

// Builds and launches the graph: memsets, init, conn, WHILE{scan, analyze, cond}, mark, count,
// chunk sums, segment scan, final, count/flag copy-out.  The instantiated graph is kept in the
// context (one per form) and launched again, with only the init and final nodes' arguments
// updated, while the sizes and scratch buffers stay the same.
template <class G, class FI, class FC, class FS, class FA, class FM, class FF>
int run_graph(be_ctx *c, int kind, G g, int64_t nblocks, int64_t nfinal, int64_t nwords, FI f_init, FC f_conn,
              FS f_scan, FA f_an, FM f_mark, FF f_final, cudaStream_t s, int64_t ninit = -1)
{
    if (ninit < 0) ninit = nblocks;   // threads of the init launch (the others run over nblocks)
    be_iter_graph &cache = c->iter_graph[kind];
    std::vector<unsigned char> key(sizeof(G) + 5 * sizeof(int64_t));
    {
        G k;
        std::memcpy(&k, &g, sizeof(G));
        blank_io(k);
        std::memcpy(key.data(), &k, sizeof(G));
        const int64_t extra[5] = {nblocks, nfinal, nwords, int64_t(reinterpret_cast<uintptr_t>(c->iter_err)), ninit};
        std::memcpy(key.data() + sizeof(G), extra, sizeof(extra));
    }
    cudaError_t e;
    if (cache.exec && cache.key == key) {
        e = set_kernel_args(cache.exec, cache.init, reinterpret_cast<void *>(f_init), nblk(ninit), g);
        if (e == cudaSuccess)
            e = set_kernel_args(cache.exec, cache.fin, reinterpret_cast<void *>(f_final), nblk(nfinal), g);
        if (e == cudaSuccess) e = cudaGraphLaunch(cache.exec, s);
        if (e != cudaSuccess) return cuda_error(c, e, "iterative graph (cached)");
        return BE_OK;
    }
    if (cache.exec) cudaGraphExecDestroy(cache.exec);
    if (cache.graph) cudaGraphDestroy(cache.graph);
    cache = be_iter_graph{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t n_init = nullptr, n_final = nullptr;
    e = cudaGraphCreate(&graph, 0);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaGraphCreate");
    cudaGraphNode_t n = nullptr, prev = nullptr;
    auto chain = [&](cudaError_t err) {
        if (err == cudaSuccess) prev = n;
        return err;
    };
    cudaMemsetParams ms = {};
    ms.dst = g.rbits;
    ms.value = 0;
    ms.elementSize = 4;
    ms.width = size_t(nwords);
    ms.height = 1;
    e = chain(cudaGraphAddMemsetNode(&n, graph, nullptr, 0, &ms));
    if (e == cudaSuccess) {
        cudaMemsetParams m2 = {};
        m2.dst = g.ctl;
        m2.value = 0;
        m2.elementSize = 4;
        m2.width = 4;
        m2.height = 1;
        e = chain(cudaGraphAddMemsetNode(&n, graph, &prev, 1, &m2));
    }
    if (e == cudaSuccess) e = chain(add_kernel(graph, &n, prev, f_init, nblk(ninit), NT, g));
    if (e == cudaSuccess) n_init = n;
    if (e == cudaSuccess && f_conn) e = chain(add_kernel(graph, &n, prev, f_conn, nblk(nblocks), NT, g));
    cudaGraphConditionalHandle h;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = chain(cudaGraphAddNode(&n, graph, &prev, 1, &cp));
        if (e == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            cudaGraphNode_t b1, b2, b3;
            e = add_kernel(body, &b1, nullptr, f_scan, nblk(nblocks), NT, g);
            if (e == cudaSuccess) e = add_kernel(body, &b2, b1, f_an, nblk(nblocks), NT, g);
            if (e == cudaSuccess) e = add_kernel(body, &b3, b2, it_cond, 1u, 1u, h, g.ctl);
        }
    }
    if (e == cudaSuccess) e = chain(add_kernel(graph, &n, prev, f_mark, nblk(nblocks), NT, g));
    if (e == cudaSuccess)
        e = chain(add_kernel(graph, &n, prev, it_count, nblk(nwords), NT, (const uint32_t *)g.rbits,
                             g.w.segcnt, nwords));
    if (e == cudaSuccess)
        e = chain(add_kernel(graph, &n, prev, k_chunk_sums, unsigned(g.w.n_chunks), unsigned(kPostThreads), g.w));
    if (e == cudaSuccess)
        e = chain(add_kernel(graph, &n, prev, k_segscan, unsigned(g.w.n_chunks), unsigned(kScanThreads), g.w));
    if (e == cudaSuccess) e = chain(add_kernel(graph, &n, prev, f_final, nblk(nfinal), NT, g));
    if (e == cudaSuccess) n_final = n;
    if (e == cudaSuccess)
        e = chain(add_kernel(graph, &n, prev, it_ncomp, 1u, 1u, g.w, (const uint32_t *)g.ctl, g.ctl + 3));
    if (e == cudaSuccess) {
        cudaMemcpy3DParms cp = {};
        cp.srcPtr = make_cudaPitchedPtr(g.ctl + 3, 4, 1, 1);
        cp.dstPtr = make_cudaPitchedPtr(c->iter_err, 4, 1, 1);
        cp.extent = make_cudaExtent(4, 1, 1);
        cp.kind = cudaMemcpyDeviceToHost;
        e = chain(cudaGraphAddMemcpyNode(&n, graph, &prev, 1, &cp));
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    if (e != cudaSuccess) {
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return cuda_error(c, e, "iterative graph");
    }
    cache.key = std::move(key);
    cache.graph = graph;
    cache.exec = exec;
    cache.init = n_init;
    cache.fin = n_final;
    return BE_OK;
}

}  // namespace

int run_iter2d(be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr,
               int32_t *out, int64_t out_pitch, cudaStream_t s)
{
    It2 g{};
    g.in = in; g.pitch = in_pitch; g.out = out; g.opitch = out_pitch;
    g.rows = rows; g.cols = cols; g.thr = thr;
    g.bw = (cols + 1) / 2; g.bh = (rows + 1) / 2;
    g.sx = ceil_log2(cols);
    const int64_t keyspace = int64_t(rows) << g.sx;
    if (keyspace >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "iterative form: %d x %d exceeds its key space", rows, cols);
    const int64_t nblocks = int64_t(g.bw) * g.bh, nwords = (keyspace + 31) / 32;
    char *lab, *mk, *conn, *rb, *ctl;
    int rc = iter_scratch(c, nblocks, 1, nwords, &lab, &mk, &conn, &rb, &ctl);
    if (rc) return rc;
    rc = c->wsiter.ensure(c, geometry_2d(), 0, nwords, 1);
    if (rc) return rc;
    g.lab = reinterpret_cast<uint32_t *>(lab); g.mk = reinterpret_cast<uint8_t *>(mk);
    g.conn = reinterpret_cast<uint8_t *>(conn); g.rbits = reinterpret_cast<uint32_t *>(rb);
    g.ctl = reinterpret_cast<uint32_t *>(ctl);
    g.w = c->wsiter.w;
    g.w.n_tiles = 0;
    g.w.queue = nullptr;
    return run_graph(c, 0, g, nblocks, int64_t(g.bw) * rows, nwords, it_init_2d, it_conn_2d, it_scan_2d,
                     it_analyze_2d, it_mark_2d, it_final_2d, s);
}

int run_iter3d(be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int thr, int32_t *out,
               cudaStream_t s)
{
    It3 g{};
    g.in = in; g.out = out; g.d0 = d0; g.d1 = d1; g.d2 = d2; g.thr = thr;
    g.b0 = (d0 + 1) / 2; g.b1 = (d1 + 1) / 2; g.b2 = (d2 + 1) / 2;
    g.s1 = ceil_log2(d1); g.s2 = ceil_log2(d2);
    const int64_t keyspace = int64_t(d0) << (g.s1 + g.s2);
    if (keyspace >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "iterative form: volume exceeds its key space");
    const int64_t nblocks = int64_t(g.b0) * g.b1 * g.b2, nwords = (keyspace + 31) / 32;
    char *lab, *mk, *conn, *rb, *ctl;
    int rc = iter_scratch(c, nblocks, 4, nwords, &lab, &mk, &conn, &rb, &ctl);
    if (rc) return rc;
    rc = c->wsiter.ensure(c, geometry_2d(), 0, nwords, 1);
    if (rc) return rc;
    g.lab = reinterpret_cast<uint32_t *>(lab); g.mk = reinterpret_cast<uint8_t *>(mk);
    g.conn = reinterpret_cast<uint32_t *>(conn); g.rbits = reinterpret_cast<uint32_t *>(rb);
    g.ctl = reinterpret_cast<uint32_t *>(ctl);
    g.w = c->wsiter.w;
    g.w.n_tiles = 0;
    g.w.queue = nullptr;
    return run_graph(c, 1, g, nblocks, int64_t(d0) * d1 * d2, nwords, it_init_3d, it_conn_3d, it_scan_3d,
                     it_analyze_3d, it_mark_3d, it_final_3d, s);
}

int run_lbeq2d(be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr,
               int conn8, int32_t *out, int64_t out_pitch, cudaStream_t s)
{
    Lq2 g{};
    g.in = in; g.pitch = in_pitch; g.out = out; g.opitch = out_pitch;
    g.rows = rows; g.cols = cols; g.thr = thr; g.conn8 = conn8;
    g.sx = ceil_log2(cols);
    const int64_t keyspace = int64_t(rows) << g.sx;
    if (keyspace >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "label equivalence: %d x %d exceeds its key space", rows, cols);
    const int64_t n = int64_t(rows) * cols, nwords = (keyspace + 31) / 32;
    char *lab, *mk, *conn, *rb, *ctl;
    int rc = iter_scratch(c, n, 0, nwords, &lab, &mk, &conn, &rb, &ctl);
    if (rc) return rc;
    rc = c->wsiter.ensure(c, geometry_2d(), 0, nwords, 1);
    if (rc) return rc;
    g.lab = reinterpret_cast<uint32_t *>(lab); g.rbits = reinterpret_cast<uint32_t *>(rb);
    g.ctl = reinterpret_cast<uint32_t *>(ctl);
    g.w = c->wsiter.w;
    g.w.n_tiles = 0;
    g.w.queue = nullptr;
    return run_graph(c, 2, g, n, n, nwords, lq_init_2d, (void (*)(Lq2)) nullptr, lq_scan_2d, lq_analyze_2d,
                     lq_mark_2d, lq_final_2d, s);
}

int run_lbeq3d(be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int thr, int32_t *out,
               cudaStream_t s)
{
    Lq3 g{};
    g.in = in; g.out = out; g.d0 = d0; g.d1 = d1; g.d2 = d2; g.thr = thr;
    g.s1 = ceil_log2(d1); g.s2 = ceil_log2(d2);
    const int64_t keyspace = int64_t(d0) << (g.s1 + g.s2);
    if (keyspace >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "label equivalence: volume exceeds its key space");
    const int64_t n = int64_t(d0) * d1 * d2, nwords = (keyspace + 31) / 32;
    char *lab, *mk, *conn, *rb, *ctl;
    int rc = iter_scratch(c, n, 0, nwords, &lab, &mk, &conn, &rb, &ctl);
    if (rc) return rc;
    rc = c->wsiter.ensure(c, geometry_2d(), 0, nwords, 1);
    if (rc) return rc;
    g.lab = reinterpret_cast<uint32_t *>(lab); g.rbits = reinterpret_cast<uint32_t *>(rb);
    g.ctl = reinterpret_cast<uint32_t *>(ctl);
    g.w = c->wsiter.w;
    g.w.n_tiles = 0;
    g.w.queue = nullptr;
    return run_graph(c, 3, g, n, n, nwords, lq_init_3d, (void (*)(Lq3)) nullptr, lq_scan_3d, lq_analyze_3d,
                     lq_mark_3d, lq_final_3d, s);
}

int run_runeq2d(be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr, int conn8,
                int32_t *out, int64_t out_pitch, cudaStream_t s)
{
    Re2 g{};
    g.in = in; g.pitch = in_pitch; g.out = out; g.opitch = out_pitch;
    g.rows = rows; g.cols = cols; g.thr = thr; g.conn8 = conn8 ? 1 : 0;
    g.sx = ceil_log2(cols);
    g.words = (cols + 31) / 32;
    g.rmax = (cols + 1) / 2;
    const int64_t keyspace = int64_t(rows) << g.sx;
    if (keyspace >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "run equivalence: %d x %d exceeds its key space", rows, cols);
    const int64_t nruns = int64_t(rows) * g.rmax, nwords = (keyspace + 31) / 32;
    const int64_t rw = int64_t(rows) * g.words;
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    const size_t extra = 3 * al(size_t(rw) * 4) + al(size_t(rows) * 4) + 2 * al(size_t(nruns) * 4);
    char *lab, *mk, *nb, *rb, *ctl, *ex;
    int rc = iter_scratch(c, nruns, sizeof(uint4), nwords, &lab, &mk, &nb, &rb, &ctl, extra, &ex);
    if (rc) return rc;
    rc = c->wsiter.ensure(c, geometry_2d(), 0, nwords, 1);
    if (rc) return rc;
    g.lab = reinterpret_cast<uint32_t *>(lab);
    g.nb = reinterpret_cast<uint4 *>(nb);
    g.rbits = reinterpret_cast<uint32_t *>(rb);
    g.ctl = reinterpret_cast<uint32_t *>(ctl);
    g.fgb = reinterpret_cast<uint32_t *>(ex); ex += al(size_t(rw) * 4);
    g.stb = reinterpret_cast<uint32_t *>(ex); ex += al(size_t(rw) * 4);
    g.spre = reinterpret_cast<uint32_t *>(ex); ex += al(size_t(rw) * 4);
    g.nrun = reinterpret_cast<uint32_t *>(ex); ex += al(size_t(rows) * 4);
    g.rl = reinterpret_cast<int32_t *>(ex); ex += al(size_t(nruns) * 4);
    g.rr = reinterpret_cast<int32_t *>(ex);
    g.w = c->wsiter.w;
    g.w.n_tiles = 0;
    g.w.queue = nullptr;
    return run_graph(c, 4, g, nruns, int64_t(rows) * ((cols + 3) / 4), nwords, re_rows, re_nbr, re_scan, re_analyze,
                     re_mark, re_final, s, int64_t(rows) * 32);
}

}  // namespace be

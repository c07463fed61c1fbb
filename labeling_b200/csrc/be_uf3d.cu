// be_uf3d.cu -- 3D Block-Equivalence labeling, union-find form (26-connectivity, 2x2x2 blocks).
//
// Replaces the reference's BLEQ3D_Init / BLEQ3D_Scan / BLEQ3D_Analyze / BLEQ3D_SetFinalLabels
// (LabelingAlgs.cl:740-979) and their host loop (LabelingAlgs.cpp:1443-1536) with the same
// four-launch structure as the 2D pipeline (be_uf2d_impl.cuh):
//
//   k_tile_local_3d   one CTA per 16 x 32 x 64-voxel tile (8 x 16 x 32 blocks): 16-byte loads,
//                     voxel-class words per block row, runs along d2 and their links to the four
//                     preceding rows by bit operations, a shared-memory union-find over runs (the
//                     run of the component's first voxel stays the root), one uint32 per block,
//                     segment root counts, a per-tile bitmap of component first voxels, border
//                     components exported as nodes.
//   k_merge_3d        global union-find over nodes across the +d0 / +d1 / +d2 tile faces; a root
//                     linked under another leaves its segment count and its tile's bitmap.
//   k_scan_link_3d    exclusive scan of the segment counts (single pass, look-back) and, in the
//                     same launch, every linked node pointed at its global root with the segment
//                     and in-segment rank of that root's first voxel resolved.
//   k_tile_write_3d   resolves canonical labels (segment prefix + rank in the bitmap row) and
//                     writes int32 voxels with 16-byte stores.
//
// Volume layout is the reference's cv::Mat 3-D order [d0][d1][d2] with d2 fastest
// (Read3DImage, main.cpp:191-203; kernel addressing x*h*d + y*d + z, LabelingAlgs.cl:974).
// Mask bit v = 4i + 2j + k is the voxel at offset (i, j, k) in (d0, d1, d2); the lowest set bit
// is the block's first voxel in raster order.
//
// Block connectivity.  Two blocks A and B = A + d are 26-connected iff A has a foreground voxel
// on its side facing B and B has one on its side facing A: along an axis with d = -1 only offset
// 0 of A and offset 1 of B can touch, along an axis with d = 0 every offset can.  This is the
// predicate the reference evaluates voxel by voxel with TEST_CONN1/2/4 (LabelingAlgs.cl:770-856).
//
// Within a tile the union-find entries carry the slot (b0, i, b1, j, b2) of a run's first voxel,
// whose order is the raster order of first voxels, and the atomicMin union keeps the smaller slot as
// the root: the root run of a component holds its first voxel.
#include "be_common.cuh"
#include "be_kernels.h"
#include "be_scan.cuh"

namespace be {

namespace {

constexpr int TB0 = T3_TB0, TB1 = T3_TB1, TB2 = T3_TB2;   // tile in blocks
constexpr int TX = 2 * TB0, TY = 2 * TB1, TZ = 2 * TB2;   // tile in voxels
constexpr int NBLK = T3_NBLK;
constexpr int NPERIM = T3_NPERIM;
constexpr int MAXB = T3_MAXB;
constexpr int NT = kT3Threads;
constexpr int RBW = TZ / 32;                // root-bitmap words per voxel row
constexpr uint32_t ROOT_FLAG = 1u << 23;

static_assert(NBLK <= (1 << 13), "tile-local block index must fit the entry payload");
static_assert(TX * TY * TZ <= (1 << 23), "tile-local key must fit the entry payload");
static_assert(NPERIM < 65536 && MAXB < 4096, "border encodings");

__device__ __forceinline__ int blk(int b0, int b1, int b2) { return (b0 * TB1 + b1) * TB2 + b2; }

// Highest set bit of x (x != 0).
__device__ __forceinline__ uint32_t hibit3(uint32_t x) { return 31u - __clz(x); }

// Tile-local key of the first voxel of a block.
__device__ __forceinline__ uint32_t local_key(int b, uint32_t m)
{
    const int v = __ffs(m) - 1;
    const int b2 = b % TB2, b1 = (b / TB2) % TB1, b0 = b / (TB1 * TB2);
    const int X = 2 * b0 + (v >> 2), Y = 2 * b1 + ((v >> 1) & 1), Z = 2 * b2 + (v & 1);
    return uint32_t((X * TY + Y) * TZ + Z);
}

// Border faces: 0 = -d0, 1 = +d0, 2 = -d1, 3 = +d1, 4 = -d2, 5 = +d2.
__device__ __forceinline__ int face_base(int f)
{
    constexpr int sz[6] = {TB1 * TB2, TB1 * TB2, TB0 * TB2, TB0 * TB2, TB0 * TB1, TB0 * TB1};
    int b = 0;
    for (int i = 0; i < f; ++i) b += sz[i];
    return b;
}

// The four voxels of a block on face f, as bits (a*2 + b) over the two tangent axes in order.
__device__ __forceinline__ uint32_t face_bits(uint32_t m, int f)
{
    // Mask bit v = 4i + 2j + k; the face's four voxels in the order (first tangent, second).
    const uint32_t s = uint32_t(f & 1);
    switch (f >> 1) {
    case 0: return (m >> (4 * s)) & 0xFu;                                          // (j, k)
    case 1: return ((m >> (2 * s)) & 3u) | (((m >> (4 + 2 * s)) & 3u) << 2);       // (i, k)
    default:                                                                        // (i, j)
        return ((m >> s) & 1u) | (((m >> (2 + s)) & 1u) << 1) | (((m >> (4 + s)) & 1u) << 2) |
               (((m >> (6 + s)) & 1u) << 3);
    }
}

// Selector over face bits (a*2 + b) for the tangent offsets (da, db).
__device__ __forceinline__ uint32_t face_sel(int da, int db)
{
    const uint32_t sa = da < 0 ? 0x3u : da > 0 ? 0xCu : 0xFu;
    const uint32_t sb = db < 0 ? 0x5u : db > 0 ? 0xAu : 0xFu;
    return sa & sb;
}

struct TileGeo {
    int tx0, tx1, tx2;      // tile coordinates
    int x0, y0, z0;         // first voxel
    int nx, ny, nz;         // valid voxels
    int n0, n1, n2;         // valid blocks
};

__device__ __forceinline__ TileGeo tile_geo(const Img3D &im, int64_t t)
{
    TileGeo g;
    const int64_t lt = t - im.tile_base;
    g.tx2 = int(lt % im.t2);
    g.tx1 = int((lt / im.t2) % im.t1);
    g.tx0 = int(lt / (int64_t(im.t2) * im.t1));
    g.x0 = g.tx0 * TX; g.y0 = g.tx1 * TY; g.z0 = g.tx2 * TZ;
    g.nx = min(TX, im.d0 - g.x0); g.ny = min(TY, im.d1 - g.y0); g.nz = min(TZ, im.d2 - g.z0);
    g.n0 = (g.nx + 1) >> 1; g.n1 = (g.ny + 1) >> 1; g.n2 = (g.nz + 1) >> 1;
    return g;
}

// Block position of border position p (face f, index q), when valid for this tile.
__device__ __forceinline__ bool perim_pos3(int p, const TileGeo &g, int &f, int &b0, int &b1, int &b2)
{
    constexpr int F0 = TB1 * TB2, F1 = TB0 * TB2;   // positions on a d0 face, on a d1 face
    int q;
    if (p < 2 * F0) { f = p >= F0; q = p - f * F0; }
    else if (p < 2 * F0 + 2 * F1) { const int r = p - 2 * F0; f = 2 + (r >= F1); q = r - (f - 2) * F1; }
    else { const int r = p - 2 * F0 - 2 * F1; f = 4 + (r >= TB0 * TB1); q = r - (f - 4) * TB0 * TB1; }
    const int axis = f >> 1, hi = f & 1;
    if (axis == 0) { b0 = hi ? g.n0 - 1 : 0; b1 = q / TB2; b2 = q % TB2; }
    else if (axis == 1) { b1 = hi ? g.n1 - 1 : 0; b0 = q / TB2; b2 = q % TB2; }
    else { b2 = hi ? g.n2 - 1 : 0; b0 = q / TB1; b1 = q % TB1; }
    return b0 < g.n0 && b1 < g.n1 && b2 < g.n2;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Tile-local labeling.  One thread per block row along d2: the tile is TB2 = 32 blocks deep, so a
// row is one 32-bit word per voxel class (v = 4i + 2j + k, the voxel's offsets in its block).
// Faces, runs along d2, run starts and the links to the four preceding rows are bit operations;
// only runs enter the union-find, ordered by the raster position of their first voxel.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int NT1 = kT3LocalThreads;   // threads of the tile-local kernel: one per block row
constexpr int MQ1 = 1024;          // union-queue capacity (more are merged in place)
static_assert(TB2 == 32, "a block row along d2 is one 32-bit word");
static_assert(NBLK <= 4096, "run starts must fit 12 bits");

// Word of the blocks whose side toward (dx, dy, dz) holds a foreground voxel: the OR of the
// classes with offset 0 along an axis where d < 0, offset 1 where d > 0.
template <int DX, int DY, int DZ>
__device__ __forceinline__ uint32_t face_word(const uint32_t (&c)[8])
{
    uint32_t r = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const int i = v >> 2, j = (v >> 1) & 1, k = v & 1;
        if ((DX < 0 && i) || (DX > 0 && !i) || (DY < 0 && j) || (DY > 0 && !j) || (DZ < 0 && k) || (DZ > 0 && !k))
            continue;
        r |= c[v];
    }
    return r;
}

// Slot of a block with first voxel offsets (i, j): the raster order of first voxels is the order
// of (b0, i, b1, j, b2) (b2 decides last: blocks of one row and class differ only there).
__device__ __forceinline__ uint32_t slot3(int b0, int i, int b1, int j, int b2)
{
    return uint32_t((((b0 * 2 + i) * TB1 + b1) * 2 + j) * TB2 + b2);
}

__device__ __forceinline__ uint32_t slot_block(uint32_t slot)
{
    const uint32_t b2 = slot % TB2, b1 = (slot / (2 * TB2)) % TB1, b0 = slot / (4 * TB2 * TB1);
    return (b0 * TB1 + b1) * TB2 + b2;
}

// Shared-memory position of block x's union-find entry: the low five bits (the block's place along
// d2) are XOR-ed with its row, so that the 32 lanes of a warp -- 32 rows walking the same position
// -- reach 32 different banks.  Entries still name blocks by their plain index.
__device__ __forceinline__ uint32_t sw3(uint32_t x) { return x ^ ((x >> 5) & 31u); }

// Union-find over run starts, the slot carried in the entry: (slot << 12) | parent.  The find
// (path halving) returns the root and the root's own entry as read (the union compares the two).
__device__ __forceinline__ uint32_t efind3_e(uint32_t *P, uint32_t x, uint32_t &ev)
{
    uint32_t v = P[sw3(x)];
    while ((v & 0xFFFu) != x) {
        const uint32_t y = v & 0xFFFu;
        const uint32_t vg = P[sw3(y)];
        if ((vg & 0xFFFu) != y) P[sw3(x)] = vg;
        x = y;
        v = vg;
    }
    ev = v;
    return x;
}

__device__ __forceinline__ void eunion3(uint32_t *P, uint32_t a, uint32_t b)
{
    for (;;) {
        uint32_t ea, eb;
        a = efind3_e(P, a, ea);
        b = efind3_e(P, b, eb);
        if (a == b) return;
        if (ea < eb) {
            const uint32_t old = atomicMin(&P[sw3(b)], ea);
            if ((old & 0xFFFu) == b) return;
            b = old & 0xFFFu;
        } else {
            const uint32_t old = atomicMin(&P[sw3(a)], eb);
            if ((old & 0xFFFu) == a) return;
            a = old & 0xFFFu;
        }
    }
}

// Bits 0..3 of x -> bit 0 of bytes 0..3.
__device__ __forceinline__ uint32_t spread4b(uint32_t x) { return ((x & 0xFu) * 0x00204081u) & 0x01010101u; }

// Byte-wise x > thr (bit 7 of each byte); K = 0x7F - (thr & 0x7F) per byte, hi = thr >= 128.
__device__ __forceinline__ uint32_t gt_bytes3(uint32_t x, uint32_t K, bool hi)
{
    const uint32_t s = (x & 0x7F7F7F7Fu) + K;
    return (hi ? (x & s) : (x | s)) & 0x80808080u;
}
__device__ __forceinline__ uint32_t gather4b(uint32_t g) { return (g * 0x00204081u) >> 28; }

// 16 voxels along d2 -> foreground bits of the even (k = 0) and odd (k = 1) voxels: 8 blocks.
__device__ __forceinline__ void split16b(uint4 v, uint32_t K, bool hi, uint32_t &ev, uint32_t &od)
{
    ev = gather4b(gt_bytes3(__byte_perm(v.x, v.y, 0x6420), K, hi)) |
         (gather4b(gt_bytes3(__byte_perm(v.z, v.w, 0x6420), K, hi)) << 4);
    od = gather4b(gt_bytes3(__byte_perm(v.x, v.y, 0x7531), K, hi)) |
         (gather4b(gt_bytes3(__byte_perm(v.z, v.w, 0x7531), K, hi)) << 4);
}

}  // namespace

__global__ void __launch_bounds__(NT1, kT3LocalPerSM) k_tile_local_3d(ImgList3D L, Work w)
{
    grid_dep_release();   // the merge launch may take free SMs during this grid's last wave
    if (blockIdx.x == 0 && threadIdx.x == 0) {   // a new epoch for the segment scan of this run
        w.epoch[0] += 1u;
        w.epoch[1] = 0u;
    }
    __shared__ uint32_t P[NBLK];               // run starts: (slot << 12) | parent
    __shared__ __align__(16) uint8_t M[NBLK];  // block masks
    __shared__ uint32_t CW[8][NT1];            // class words of every row
    __shared__ uint32_t WHZ[NT1], WS[NT1];     // joins along d2, run starts
    __shared__ uint32_t BF[NBLK / 32];
    __shared__ uint32_t BP[NBLK / 32];
    __shared__ uint32_t MQ[MQ1];               // union queue: (block_a << 16) | block_b
    static_assert(TX * TY * RBW <= MQ1, "the root bitmap fits the queue's memory");
    uint32_t *const RB = MQ;                   // root bitmap (after the unions)
    __shared__ uint32_t mqn[4];                // queue counts of the union rounds
    __shared__ uint32_t tmp[NT1 / 32 + 1];
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x;
    const int b0 = tid / TB1, b1 = tid % TB1;
    const uint32_t rowb = uint32_t(tid) * TB2;   // block index of the row's first block
    uint32_t *lab = reinterpret_cast<uint32_t *>(w.lab);
    ItemLoop loop{w.queue ? w.queue + 0 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
        const uint32_t K = (0x7Fu - (uint32_t(im.thr) & 0x7Fu)) * 0x01010101u;
        const bool hi = im.thr >= 128;
        const int64_t rs0 = int64_t(im.d1) * im.d2;   // stride of d0 in voxels

        BF[tid] = 0;
        if (tid < 4) mqn[tid] = 0;

        // Phase A: class words, runs along d2, run slots.
        uint32_t c[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) c[v] = 0;
        if (b0 < g.n0 && b1 < g.n1) {
#pragma unroll
            for (int ij = 0; ij < 4; ++ij) {
                const int i = ij >> 1, j = ij & 1;
                const int X = 2 * b0 + i, Y = 2 * b1 + j;
                if (X >= g.nx || Y >= g.ny) continue;
                const uint8_t *row = im.in + (g.x0 + X) * rs0 + int64_t(g.y0 + Y) * im.d2 + g.z0;
                uint32_t ev = 0, od = 0;
                if (g.nz == TZ && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
                    const uint4 *pv = reinterpret_cast<const uint4 *>(row);
                    uint4 q[4];
#pragma unroll
                    for (int h = 0; h < 4; ++h) q[h] = __ldg(pv + h);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        uint32_t e8, o8;
                        split16b(q[h], K, hi, e8, o8);
                        ev |= e8 << (8 * h);
                        od |= o8 << (8 * h);
                    }
                } else {
                    for (int z = 0; z < g.nz; ++z) {
                        const uint32_t bit = uint32_t(row[z] > im.thr) << (z >> 1);
                        if (z & 1) od |= bit;
                        else ev |= bit;
                    }
                }
                c[4 * i + 2 * j] = ev;
                c[4 * i + 2 * j + 1] = od;
            }
        }
        const uint32_t Fw = c[0] | c[1] | c[2] | c[3] | c[4] | c[5] | c[6] | c[7];
        const uint32_t hz = face_word<0, 0, 1>(c) & (face_word<0, 0, -1>(c) >> 1);   // k joined to k + 1
        const uint32_t hl = hz << 1;                                               // k joined to k - 1
        const uint32_t S = Fw & ~hl;
#pragma unroll
        for (int v = 0; v < 8; ++v) CW[v][tid] = c[v];
        WHZ[tid] = hz;
        WS[tid] = S;
        {
            uint32_t mw[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                uint32_t m = 0;
#pragma unroll
                for (int v = 0; v < 8; ++v) m |= spread4b(c[v] >> (4 * q)) << v;
                mw[q] = m;
            }
            uint4 *md = reinterpret_cast<uint4 *>(&M[rowb]);
            md[0] = make_uint4(mw[0], mw[1], mw[2], mw[3]);
            md[1] = make_uint4(mw[4], mw[5], mw[6], mw[7]);
        }
        __syncthreads();

        // Phase B: links to the four preceding rows (d0-1 with d1-1 / d1 / d1+1, and d0 with
        // d1-1), each with offsets dz = -1 / 0 / +1 along d2.  As in 2D, a link is dropped when
        // an earlier one (further along d2, or dz = 0 before dz = +-1 at the same block) joins the
        // same two runs.
        uint32_t LN[4], LW[4], LE[4];
        int UR[4];
#pragma unroll
        for (int nr = 0; nr < 4; ++nr) {
            const int dx = nr < 3 ? -1 : 0, dy = nr < 3 ? nr - 1 : -1;
            const int r0 = b0 + dx, r1 = b1 + dy;
            uint32_t N = 0, NW = 0, NE = 0;
            int ur = 0;
            if (Fw && r0 >= 0 && r1 >= 0 && r1 < TB1) {
                ur = r0 * TB1 + r1;
                uint32_t u[8];
#pragma unroll
                for (int v = 0; v < 8; ++v) u[v] = CW[v][ur];
                uint32_t A0, Am, Ap, B0, Bm, Bp;   // own sides toward dz = 0/-1/+1, neighbour's opposite sides
                if (nr == 0) {
                    A0 = face_word<-1, -1, 0>(c); Am = face_word<-1, -1, -1>(c); Ap = face_word<-1, -1, 1>(c);
                    B0 = face_word<1, 1, 0>(u); Bm = face_word<1, 1, 1>(u); Bp = face_word<1, 1, -1>(u);
                } else if (nr == 1) {
                    A0 = face_word<-1, 0, 0>(c); Am = face_word<-1, 0, -1>(c); Ap = face_word<-1, 0, 1>(c);
                    B0 = face_word<1, 0, 0>(u); Bm = face_word<1, 0, 1>(u); Bp = face_word<1, 0, -1>(u);
                } else if (nr == 2) {
                    A0 = face_word<-1, 1, 0>(c); Am = face_word<-1, 1, -1>(c); Ap = face_word<-1, 1, 1>(c);
                    B0 = face_word<1, -1, 0>(u); Bm = face_word<1, -1, 1>(u); Bp = face_word<1, -1, -1>(u);
                } else {
                    A0 = face_word<0, -1, 0>(c); Am = face_word<0, -1, -1>(c); Ap = face_word<0, -1, 1>(c);
                    B0 = face_word<0, 1, 0>(u); Bm = face_word<0, 1, 1>(u); Bp = face_word<0, 1, -1>(u);
                }
                const uint32_t uhz = WHZ[ur], uhl = uhz << 1;
                const uint32_t n0 = A0 & B0, nw = Am & (Bm << 1), ne = Ap & (Bp >> 1);
                const uint32_t Nsh = n0 << 1, NEsh = ne << 1;
                N = n0 & ~(hl & ((Nsh & uhl) | NEsh));
                NW = nw & ~((n0 & uhl) | (hl & Nsh));
                NE = ne & ~((n0 & uhz) | (hl & NEsh & uhz));
            }
            LN[nr] = N;
            LW[nr] = NW;
            LE[nr] = NE;
            UR[nr] = ur;
        }
        auto start_of = [&](uint32_t b) -> uint32_t {
            return (b & ~31u) + hibit3(WS[b >> 5] & ((2u << (b & 31u)) - 1u));
        };
        // Every run of this row gets its entry.  A run with a link into the preceding layer (d0 - 1,
        // whose slots are all smaller than this row's) takes the first one as its parent by a plain
        // store; the entry holds key 0, the smallest value, so no atomicMin of a union changes it and
        // unions walk on to the parent (only a root's key is ever compared).  These links leave the
        // queue.  Links within the same layer (d1 - 1) may go to larger slots and stay unions.  Any
        // other run is a root for now: (slot << 12) | itself, the slot being that of its first voxel.
        // (Pointer jumping over the forest before the unions was measured slower.)
        {
            const uint32_t H00 = c[0] | c[1], H01 = c[2] | c[3], H10 = c[4] | c[5], H11 = c[6] | c[7];
            uint32_t ss = S;
            while (ss) {
                const uint32_t s0 = __ffs(ss) - 1;
                ss &= ss - 1;
                const uint32_t brk = ~hz & (~0u << s0);
                const uint32_t e = brk ? uint32_t(__ffs(brk) - 1) : 31u;
                const uint32_t span = (~0u << s0) & (0xFFFFFFFFu >> (31u - e));
                const uint32_t x = rowb + s0;
                bool found = false;
#pragma unroll
                for (int nr = 0; nr < 3; ++nr) {
                    const uint32_t lk = (LN[nr] | LW[nr] | LE[nr]) & span;
                    if (found || !lk) continue;
                    found = true;
                    const uint32_t k = __ffs(lk) - 1, bit = 1u << k;
                    const uint32_t ubase = uint32_t(UR[nr]) * TB2;
                    uint32_t tgt;
                    if (LN[nr] & bit) {
                        tgt = ubase + k;
                        LN[nr] &= ~bit;
                    } else if (LW[nr] & bit) {
                        tgt = ubase + k - 1;
                        LW[nr] &= ~bit;
                    } else {
                        tgt = ubase + k + 1;
                        LE[nr] &= ~bit;
                    }
                    P[sw3(x)] = start_of(tgt);   // key 0
                }
                if (!found) {
                    int i, j;
                    uint32_t m;
                    if (H00 & span) { i = 0; j = 0; m = H00 & span; }
                    else if (H01 & span) { i = 0; j = 1; m = H01 & span; }
                    else if (H10 & span) { i = 1; j = 0; m = H10 & span; }
                    else { i = 1; j = 1; m = H11 & span; }
                    P[sw3(x)] = (slot3(b0, i, b1, j, __ffs(m) - 1) << 12) | x;
                }
            }
        }
        __syncthreads();
        // The remaining links are unions, queued and merged by every lane, one neighbour row per
        // round; a round whose links overflow the queue takes further passes through it (the links
        // with positions [base, base + MQ1) each), so the overflow is shared by every lane too.
#pragma unroll
        for (int round = 0; round < 4; ++round) {
            const uint32_t n = __popc(LN[round]) + __popc(LW[round]) + __popc(LE[round]);
            const uint32_t pos0 = warp_reserve(&mqn[round], n);
            const uint32_t ubase = uint32_t(UR[round]) * TB2;
            auto each_link = [&](auto &&fn) {
                uint32_t pos = pos0;
                uint32_t todo = LN[round] | LW[round] | LE[round];
                while (todo) {
                    const uint32_t k = __ffs(todo) - 1;
                    todo &= todo - 1;
                    const uint32_t bit = 1u << k;
                    const uint32_t a = rowb + k;
                    if (LN[round] & bit) fn(pos++, a, ubase + k);
                    if (LW[round] & bit) fn(pos++, a, ubase + k - 1);
                    if (LE[round] & bit) fn(pos++, a, ubase + k + 1);
                }
            };
            if (pos0 < uint32_t(MQ1))
                each_link([&](uint32_t pos, uint32_t a, uint32_t b) {
                    if (pos < uint32_t(MQ1)) MQ[pos] = (a << 16) | b;
                });
            __syncthreads();
            const uint32_t total = mqn[round];
            for (uint32_t base = 0; base < total; base += MQ1) {
                if (base) {
                    if (pos0 + n > base && pos0 < base + MQ1)
                        each_link([&](uint32_t pos, uint32_t a, uint32_t b) {
                            if (pos >= base && pos < base + MQ1) MQ[pos - base] = (a << 16) | b;
                        });
                    __syncthreads();
                }
                const uint32_t nq = min(total - base, uint32_t(MQ1));
                // Contiguous runs of the queue per thread, as in 2D.
                const uint32_t per = (nq + NT1 - 1) / NT1, lo = min(nq, uint32_t(tid) * per), hi = min(nq, lo + per);
                for (uint32_t q = lo; q < hi; ++q) eunion3(P, start_of(MQ[q] >> 16), start_of(MQ[q] & 0xFFFFu));
                __syncthreads();
            }
        }

        // The root bitmap lives in the queue's memory from here on (the unions are done).
        for (int i = tid; i < TX * TY * RBW; i += NT1) RB[i] = 0;
        __syncthreads();
        // Phase C: every run start of this row is pointed straight at its root (a read-only walk,
        // then the root's entry stored in the start's own entry, as in 2D); roots mark their first
        // voxel.
        {
            uint32_t ss = S;
            while (ss) {
                const uint32_t x = rowb + (__ffs(ss) - 1);
                ss &= ss - 1;
                uint32_t root = x, ev = P[sw3(x)];
                for (int it = 0; (ev & 0xFFFu) != root && it < NBLK; ++it) {   // acyclic: the cap never binds
                    root = ev & 0xFFFu;
                    ev = P[sw3(root)];
                }
                if (root != x) P[sw3(x)] = ev;
                if (root != x) continue;
                const uint32_t rb = slot_block(ev >> 12);
                const uint32_t key = local_key(int(rb), M[rb]);
                const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
                if (GUARD(w, key < uint32_t(TX * TY * TZ), 101, key))
                    atomicOr(&RB[(X * TY + Y) * RBW + (Z >> 5)], 1u << (Z & 31));
            }
        }
        // Block entries: the root block of a component carries ROOT_FLAG | its first-voxel key,
        // every other block its root block.  (Runs do not cross rows: every start read here is
        // this thread's own.)
        {
            uint32_t cur = 0;
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                const uint32_t mm = *reinterpret_cast<const uint32_t *>(&M[rowb + 4 * h]);
                uint32_t e[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int k = 4 * h + q;
                    if ((S >> k) & 1u) cur = slot_block(P[sw3(rowb + k)] >> 12);
                    const uint32_t m = (mm >> (8 * q)) & 0xFFu;
                    uint32_t v = 0;
                    if (m) {
                        v = (m << 24) | cur;
                        if (cur == rowb + uint32_t(k)) v = (m << 24) | ROOT_FLAG | local_key(int(cur), m);
                    }
                    e[q] = v;
                }
                reinterpret_cast<uint4 *>(lab + t * NBLK + rowb)[h] = make_uint4(e[0], e[1], e[2], e[3]);
            }
        }
        __syncthreads();   // root bitmap complete; every run start points at its root

        // Phase D: root bitmap and segment counts out, border nodes.
        for (int i = tid; i < TX * TY * RBW; i += NT1) w.rbits[t * (TX * TY * RBW) + i] = RB[i];
        for (int r = tid; r < TX * TY; r += NT1) {
            const int X = r / TY, Y = r % TY;
            if (X >= g.nx || Y >= g.ny) continue;
            uint32_t cnt = 0;
#pragma unroll
            for (int k = 0; k < RBW; ++k) cnt += __popc(RB[r * RBW + k]);
            const int64_t si = im.seg_base + (int64_t(g.x0 + X) * im.d1 + (g.y0 + Y)) * im.t2 + g.tx2;
            if (GUARD(w, si >= 0 && si < w.n_segs, 104, si)) w.segcnt[si] = uint8_t(cnt);
        }
        auto root_block = [&](int b) -> uint32_t {
            const uint32_t row = uint32_t(b) >> 5, k = uint32_t(b) & 31u;
            const uint32_t st = hibit3(WS[row] & ((2u << k) - 1u));
            return slot_block(P[sw3((row << 5) + st)] >> 12);
        };
        // Each border position's root block and face bits, kept in registers for the entries below
        // ((root << 4) | face bits, 16 bits each; 0 stands for an empty position -- a root block 0
        // with no face voxel gives entry 0 as well).
        constexpr int KP = NPERIM / NT1;
        static_assert(NPERIM % NT1 == 0, "border positions per thread");
        uint32_t pc[(KP + 1) / 2];
#pragma unroll
        for (int k = 0; k < KP; ++k) {
            const int p = tid + k * NT1;
            int f, pb0, pb1, pb2;
            uint32_t c = 0;
            if (perim_pos3(p, g, f, pb0, pb1, pb2)) {
                const int b = blk(pb0, pb1, pb2);
                const uint32_t m = M[b];
                if (m) {
                    const uint32_t rb = root_block(b);
                    atomicOr(&BF[rb >> 5], 1u << (rb & 31));
                    c = (rb << 4) | face_bits(m, f);
                }
            }
            if (k & 1) pc[k >> 1] |= c << 16;
            else pc[k >> 1] = c;
        }
        __syncthreads();
        uint32_t nb;
        const uint32_t pre = block_exscan<NT1>(__popc(BF[tid]), tmp, &nb);
        BP[tid] = pre;
        __syncthreads();
        {
            uint32_t bits = BF[tid];
            uint32_t j = pre;
            while (bits) {
                const int bit = __ffs(bits) - 1;
                bits &= bits - 1;
                const uint32_t rb = tid * 32 + bit;
                const uint32_t key = local_key(int(rb), M[rb]);
                if (!GUARD(w, key < uint32_t(TX * TY * TZ) && j < uint32_t(MAXB), 102, (uint64_t(j) << 32) | key))
                    break;
                const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
                const int64_t node = t * MAXB + j;
                const uint32_t vkey = uint32_t((int64_t(g.x0 + X) * im.d1 + (g.y0 + Y)) * im.d2 + (g.z0 + Z));
                w.nroot[node] = uint16_t(rb);
                w.gp[node] = gentry(vkey, uint32_t(node));
                ++j;
            }
        }
#pragma unroll
        for (int k = 0; k < KP; ++k) {
            const uint32_t c = (pc[k >> 1] >> (16 * (k & 1))) & 0xFFFFu;
            uint16_t ent = 0;
            if (c) {
                const uint32_t rb = c >> 4;
                const uint32_t j = BP[rb >> 5] + __popc(BF[rb >> 5] & ((1u << (rb & 31)) - 1u));
                ent = uint16_t((j << 4) | (c & 15u));
            }
            w.perim[t * NPERIM + tid + k * NT1] = ent;
        }
        if (tid == 0) w.nb[t] = nb;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Cross-tile merge over the +d0, +d1 and +d2 faces.
// ---------------------------------------------------------------------------------------------
namespace {

// Where the voxel with raster key `key` of image im sits: its tile, the root-bitmap word and bit of
// it in that tile, and its segment.
struct KeyPos {
    int64_t tile, word, seg;
    uint32_t bit;
};
__device__ __forceinline__ KeyPos key_pos(const Img3D &im, uint32_t key)
{
    // Keys index one volume (< 2^32 voxels): 32-bit division suffices.
    const uint32_t row = key / uint32_t(im.d2), Z = key - row * uint32_t(im.d2);
    const uint32_t X = row / uint32_t(im.d1), Y = row - X * uint32_t(im.d1);
    const uint32_t q0 = X / TX, q1 = Y / TY, q2 = Z / TZ;
    KeyPos kp;
    kp.tile = im.tile_base + (int64_t(q0) * im.t1 + q1) * im.t2 + q2;
    const uint32_t lx = X % TX, ly = Y % TY, lz = Z % TZ;
    kp.word = kp.tile * (TX * TY * RBW) + int64_t((lx * TY + ly) * RBW + (lz >> 5));
    kp.bit = lz & 31u;
    kp.seg = im.seg_base + int64_t(row) * im.t2 + q2;
    return kp;
}

// Union of two nodes of one volume; the root linked under the other leaves its segment's root
// count and its tile's root bitmap.
__device__ void gunion3d(const Img3D &im, Work &w, uint32_t a, uint32_t b)
{
    gunion_keyed(w.gp, a, b, [&](uint32_t key) {
        const KeyPos kp = key_pos(im, key);
        dec_u8(w.segcnt, kp.seg);
        atomicAnd(w.rbits + kp.word, ~(1u << kp.bit));
    });
}

}  // namespace

// Cross-tile merge over the +d0, +d1 and +d2 faces.  The border entries of the blocks across
// each + face (the next tile's - face, widened by one block on every side into the diagonal
// tiles) are staged in shared memory once per tile, so each face block checks its nine
// neighbours without index arithmetic or global loads.  A CTA-local union-find over this tile's
// nodes and the staged positions then filters the pairs: only a pair that joins two local sets
// goes on to the global union-find (from a shared queue, once the tile's pairs are all seen); a
// dense volume that crosses a face with one component in hundreds of blocks costs a handful of
// global unions.
constexpr int kGQ3 = 256;    // queued global unions per tile (more are done at once)
constexpr int kPL3 = 576;    // listed face pairs per tile (more are checked where they are found)
constexpr int PF0 = (TB1 + 2) * (TB2 + 2);   // staged entries across the +d0 face
constexpr int PF1 = (TB0 + 2) * (TB2 + 2);   // +d1
constexpr int PF2 = (TB0 + 2) * (TB1 + 2);   // +d2
constexpr int NPF = PF0 + PF1 + PF2;
constexpr int NPLUS = TB1 * TB2 + TB0 * TB2 + TB0 * TB1;
constexpr int NSROWS = (TB1 + 2) + (TB0 + 2) + (TB0 + 2);   // staged rows over the three faces

// Face geometry along axis AX (compile-time, so nothing is indexed at run time): the two tangent
// axes in order, their tile sizes, the staged array's offset and pitch.
template <int AX> struct FaceAx {
    static constexpr int A1 = AX == 0 ? 1 : 0, A2 = AX == 2 ? 1 : 2;
    static constexpr int TA = A1 == 0 ? TB0 : TB1, TBb = A2 == 1 ? TB1 : TB2;
    static constexpr int TAX = AX == 0 ? TB0 : AX == 1 ? TB1 : TB2;
    static constexpr int EBASE = AX == 0 ? 0 : AX == 1 ? PF0 : PF0 + PF1;
    static constexpr int PITCH = TBb + 2;
    static constexpr int NPOS = TA * TBb;
    static constexpr int PBASE = AX == 0 ? 0 : AX == 1 ? TB1 * TB2 : TB1 * TB2 + TB0 * TB2;
};

__device__ __forceinline__ int pick3(int a0, int a1, int a2, int i) { return i == 0 ? a0 : i == 1 ? a1 : a2; }

// Stage entry e (0 <= e < (TA+2) * (TBb+2)) of the face along AX.
template <int AX>
__device__ __forceinline__ void stage_face(const Img3D &im, const TileGeo &g, Work &w, int e, uint32_t *nbid,
                                           uint8_t *nbf)
{
    using F = FaceAx<AX>;
    const int iu = e / F::PITCH, iv = e % F::PITCH;
    const int tcx = pick3(g.tx0, g.tx1, g.tx2, AX), tnx = pick3(im.t0, im.t1, im.t2, AX);
    const int tc1 = pick3(g.tx0, g.tx1, g.tx2, F::A1), tc2 = pick3(g.tx0, g.tx1, g.tx2, F::A2);
    const int nb1 = (pick3(im.d0, im.d1, im.d2, F::A1) + 1) >> 1, nb2 = (pick3(im.d0, im.d1, im.d2, F::A2) + 1) >> 1;
    const int g1 = tc1 * F::TA + iu - 1, g2 = tc2 * F::TBb + iv - 1;
    uint32_t id = kNone, fb = 0;
    if (tcx + 1 < tnx && g1 >= 0 && g1 < nb1 && g2 >= 0 && g2 < nb2) {
        const int t1 = g1 / F::TA, l1 = g1 - t1 * F::TA, t2 = g2 / F::TBb, l2 = g2 - t2 * F::TBb;
        int tt0, tt1, tt2;
        if (AX == 0) { tt0 = tcx + 1; tt1 = t1; tt2 = t2; }
        else if (AX == 1) { tt0 = t1; tt1 = tcx + 1; tt2 = t2; }
        else { tt0 = t1; tt1 = t2; tt2 = tcx + 1; }
        const int64_t t2i = im.tile_base + (int64_t(tt0) * im.t1 + tt1) * im.t2 + tt2;
        const int qb = l1 * F::TBb + l2;   // position on the - face: (first tangent, second tangent)
        if (GUARD(w, t2i >= 0 && t2i < w.n_tiles && qb >= 0 && qb < NPERIM, 201, t2i)) {
            const uint32_t B = w.perim[t2i * NPERIM + face_base(2 * AX) + qb];
            if (B && GUARD(w, (B >> 4) < w.nb[t2i], 203, (uint64_t(t2i) << 16) | (B >> 4))) {
                id = uint32_t(t2i * MAXB + (B >> 4));
                fb = B & 15u;
            }
        }
    }
    nbid[F::EBASE + e] = id;
    nbf[F::EBASE + e] = uint8_t(fb);
}

// This tile's + face entry at position q of the face along AX (0 when the face has no neighbour).
template <int AX>
__device__ __forceinline__ uint32_t plus_entry(const Img3D &im, const TileGeo &g, const Work &w, int64_t t, int q,
                                               int &u, int &v)
{
    using F = FaceAx<AX>;
    u = q / F::TBb;
    v = q % F::TBb;
    const int tcx = pick3(g.tx0, g.tx1, g.tx2, AX), tnx = pick3(im.t0, im.t1, im.t2, AX);
    const int n1 = pick3(g.n0, g.n1, g.n2, F::A1), n2 = pick3(g.n0, g.n1, g.n2, F::A2);
    if (tcx + 1 >= tnx || u >= n1 || v >= n2) return 0u;
    return w.perim[t * NPERIM + face_base(2 * AX + 1) + q];
}

// Tangent coordinates of position q of this tile's + face along AX.
template <int AX>
__device__ __forceinline__ void plus_uv(int q, int &u, int &v)
{
    using F = FaceAx<AX>;
    u = q / F::TBb;
    v = q % F::TBb;
}

// Staged position e of the face along AX -> (iu, iv) in the staged grid, or false when e lies in
// another face's range.
template <int AX>
__device__ __forceinline__ bool staged_pos(int e, int &iu, int &iv)
{
    using F = FaceAx<AX>;
    const int k = e - F::EBASE;
    if (k < 0 || k >= (F::TA + 2) * F::PITCH) return false;
    iu = k / F::PITCH;
    iv = k % F::PITCH;
    return true;
}

__global__ void __launch_bounds__(kT3MergeThreads, kT3MergePerSM) k_merge_3d(ImgList3D L, Work w)
{
    grid_dep_wait();
    grid_dep_release();
    __shared__ uint32_t qslot;
    __shared__ uint32_t lp[MAXB + NPF];   // local union-find: this tile's nodes, then staged positions
    __shared__ uint32_t nbid[NPF];        // global node id across the face, kNone = none
    __shared__ uint8_t nbf[NPF];          // its face bits
    __shared__ uint2 gq[kGQ3];
    __shared__ uint32_t nq;
    __shared__ uint32_t pl[kPL3];         // listed pairs: (node << 16) | staged position
    __shared__ uint32_t npl;
    __shared__ uint16_t own[NPLUS];       // this tile's + face entries (staged with the others)
    ItemLoop loop{w.queue ? w.queue + 1 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
        for (int i = threadIdx.x; i < MAXB + NPF; i += kT3MergeThreads) lp[i] = uint32_t(i);
        if (threadIdx.x == 0) {
            nq = 0;
            npl = 0;
        }
        for (int e = threadIdx.x; e < PF0; e += kT3MergeThreads) stage_face<0>(im, g, w, e, nbid, nbf);
        for (int e = threadIdx.x; e < PF1; e += kT3MergeThreads) stage_face<1>(im, g, w, e, nbid, nbf);
        for (int e = threadIdx.x; e < PF2; e += kT3MergeThreads) stage_face<2>(im, g, w, e, nbid, nbf);
        for (int q = threadIdx.x; q < NPLUS; q += kT3MergeThreads) {
            int u, v;
            if (q < FaceAx<0>::NPOS) own[q] = uint16_t(plus_entry<0>(im, g, w, t, q, u, v));
            else if (q < FaceAx<0>::NPOS + FaceAx<1>::NPOS) own[q] = uint16_t(plus_entry<1>(im, g, w, t, q - FaceAx<1>::PBASE, u, v));
            else own[q] = uint16_t(plus_entry<2>(im, g, w, t, q - FaceAx<2>::PBASE, u, v));
        }
        __syncthreads();
        // Staged positions of the same node that touch on the face are one element from here on
        // (a component crosses a face as a patch, not as scattered blocks): runs along each staged
        // row point at their first position, runs of neighbouring rows are merged where one of
        // them starts, and every staged position is then pointed straight at its root.
        for (int row = threadIdx.x; row < NSROWS; row += kT3MergeThreads) {
            int e0, n;
            if (row < FaceAx<0>::TA + 2) { e0 = FaceAx<0>::EBASE + row * FaceAx<0>::PITCH; n = FaceAx<0>::PITCH; }
            else if (row < FaceAx<0>::TA + FaceAx<1>::TA + 4) {
                e0 = FaceAx<1>::EBASE + (row - FaceAx<0>::TA - 2) * FaceAx<1>::PITCH; n = FaceAx<1>::PITCH;
            } else {
                e0 = FaceAx<2>::EBASE + (row - FaceAx<0>::TA - FaceAx<1>::TA - 4) * FaceAx<2>::PITCH; n = FaceAx<2>::PITCH;
            }
            uint32_t prev = kNone, start = 0;
            for (int k = 0; k < n; ++k) {
                const uint32_t id = nbid[e0 + k];
                if (id != prev) start = uint32_t(MAXB + e0 + k);
                lp[MAXB + e0 + k] = start;
                prev = id;
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NPF; e += kT3MergeThreads) {
            const uint32_t id = nbid[e];
            if (id == kNone) continue;
            int iu, iv, pitch;
            if (staged_pos<0>(e, iu, iv)) pitch = FaceAx<0>::PITCH;
            else if (staged_pos<1>(e, iu, iv)) pitch = FaceAx<1>::PITCH;
            else { staged_pos<2>(e, iu, iv); pitch = FaceAx<2>::PITCH; }
            if (iu == 0 || nbid[e - pitch] != id) continue;
            // One link per pair of overlapping runs: at the overlap's first column, where one of
            // the two runs starts.
            const bool xs = iv == 0 || nbid[e - 1] != id, ys = iv == 0 || nbid[e - pitch - 1] != id;
            if (xs || ys) smerge(lp, uint32_t(MAXB + e), uint32_t(MAXB + e - pitch));
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NPF; e += kT3MergeThreads)
            if (nbid[e] != kNone) sflatten(lp, uint32_t(MAXB + e));
        __syncthreads();
        // Pairs: every face position lists its connected neighbours (a bit test each) in one pass
        // over the three faces, then all lanes check the listed pairs; a pair whose two elements are
        // already one local set is implied by pairs queued before it (smerge_joined).  Pairs past
        // the list's capacity are checked by the lane that finds them.  The rest are unioned
        // globally at the end.
        auto check_pair = [&](uint32_t ja2, uint32_t e) {
            if (!smerge_joined(lp, ja2, uint32_t(MAXB) + e)) return;
            const uint32_t nA = uint32_t(t * MAXB + ja2), id = nbid[e];
            const uint32_t slot = atomicAdd(&nq, 1u);
            if (slot < uint32_t(kGQ3)) gq[slot] = make_uint2(nA, id);
            else gunion3d(im, w, nA, id);
        };
        const uint32_t nbt = w.nb[t];   // (read by the bounds checks of checked builds)
        (void)nbt;
        for (int base = 0; base < NPLUS; base += kT3MergeThreads) {
            const int p = base + int(threadIdx.x);
            int u = 0, v = 0, ebase = 0, pitch = 1;
            uint32_t A = 0;
            if (p < FaceAx<0>::NPOS) {
                plus_uv<0>(p, u, v);
                ebase = FaceAx<0>::EBASE; pitch = FaceAx<0>::PITCH;
            } else if (p < FaceAx<0>::NPOS + FaceAx<1>::NPOS) {
                plus_uv<1>(p - FaceAx<1>::PBASE, u, v);
                ebase = FaceAx<1>::EBASE; pitch = FaceAx<1>::PITCH;
            } else if (p < NPLUS) {
                plus_uv<2>(p - FaceAx<2>::PBASE, u, v);
                ebase = FaceAx<2>::EBASE; pitch = FaceAx<2>::PITCH;
            }
            if (p < NPLUS) A = own[p];
            if (A && !GUARD(w, (A >> 4) < nbt && (A >> 4) < uint32_t(MAXB), 204, (uint64_t(t) << 16) | (A >> 4)))
                A = 0;
            const uint32_t fa = A & 15u, ja = A >> 4;
            uint32_t hit = 0;   // bit 3 * (da + 1) + (db + 1): connected neighbour
            if (A) {
#pragma unroll
                for (int da = -1; da <= 1; ++da) {
#pragma unroll
                    for (int db = -1; db <= 1; ++db) {
                        if (!(fa & face_sel(da, db))) continue;
                        const int e = ebase + (u + 1 + da) * pitch + (v + 1 + db);
                        if (nbid[e] != kNone && (nbf[e] & face_sel(-da, -db))) hit |= 1u << (3 * (da + 1) + (db + 1));
                    }
                }
            }
            // Neighbours whose staged positions already share a local parent are one local set
            // (mostly one node's patch across the face): the first of them stands for the others.
            uint32_t keep = 0;
            {
                uint32_t h = hit, last0 = kNone, last1 = kNone;
                while (h) {
                    const int k = __ffs(h) - 1;
                    h &= h - 1;
                    const uint32_t a = lp[MAXB + ebase + (u + k / 3) * pitch + (v + k % 3)];
                    if (a == last0 || a == last1) continue;
                    last1 = last0;
                    last0 = a;
                    keep |= 1u << k;
                }
            }
            uint32_t pos = warp_reserve(&npl, __popc(keep));
            while (keep) {
                const int k = __ffs(keep) - 1;
                keep &= keep - 1;
                const uint32_t e = uint32_t(ebase + (u + k / 3) * pitch + (v + k % 3));
                if (pos < uint32_t(kPL3)) pl[pos] = (ja << 16) | e;
                else check_pair(ja, e);
                ++pos;
            }
        }
        __syncthreads();
        {
            const uint32_t n = min(npl, uint32_t(kPL3));
            for (uint32_t i = threadIdx.x; i < n; i += kT3MergeThreads) check_pair(pl[i] >> 16, pl[i] & 0xFFFFu);
        }
        __syncthreads();
        const uint32_t nqt = min(nq, uint32_t(kGQ3));
        for (uint32_t i = threadIdx.x; i < nqt; i += kT3MergeThreads) gunion3d(im, w, gq[i].x, gq[i].y);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Segment scan and node links, one launch: items below n_chunks scan a chunk of segment counts
// (single pass, look-back); the others resolve the linked nodes of one tile (link_tile_nodes):
// each is pointed straight at its global root, and the segment and in-segment rank of that root's
// first voxel are stored with it.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kScanThreads) k_scan_link_3d(ImgList3D L, Work w)
{
    grid_dep_wait();
    grid_dep_release();   // after the wait: the label-write launch relies on it
    __shared__ uint32_t tmp[kScanThreads / 32 + 1];
    __shared__ uint32_t sh[2];
    __shared__ uint32_t qslot;
    const int64_t n = int64_t(w.n_chunks) + w.n_tiles;
    ItemLoop loop{w.queue ? w.queue + 2 : nullptr, n};
    for (int64_t it = loop.first(&qslot); it < n; it = loop.next(it, &qslot)) {
        if (it < w.n_chunks) {
            segscan_lb_chunk<kScanThreads>(w, tmp, sh);
            continue;
        }
        const int64_t t = it - w.n_chunks;
        const Img3D im = L.get(t);
        link_tile_nodes(w, t, MAXB, [&](uint32_t key, uint32_t &seg, uint32_t &rank) {
            const KeyPos kp = key_pos(im, key);
            const uint32_t *rw = w.rbits + (kp.word & ~int64_t(RBW - 1));
            rank = __popc(rw[kp.word & (RBW - 1)] & ((1u << kp.bit) - 1u));
            for (int k = 0; k < int(kp.word & (RBW - 1)); ++k) rank += __popc(rw[k]);
            seg = uint32_t(kp.seg);
        });
    }
}

// ---------------------------------------------------------------------------------------------
// Label resolve and write.
// ---------------------------------------------------------------------------------------------
constexpr int kNLCap = 512;   // node links a write CTA stages in shared memory (later ones: from L2)

__global__ void __launch_bounds__(NT, 5) k_tile_write_3d(ImgList3D L, Work w)
{
    __shared__ __align__(16) uint32_t Ls[NBLK];
    __shared__ uint32_t LT[NBLK];
    __shared__ __align__(16) uint32_t RB[TX * TY * RBW];
    __shared__ uint32_t segb[TX * TY + 1];   // segment prefixes of the tile's voxel rows; [TX * TY]: the volume's first
    __shared__ __align__(16) uint2 NL[kNLCap];
    __shared__ uint32_t snb;
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x;
    const uint32_t *lab = reinterpret_cast<const uint32_t *>(w.lab);
    static_assert(NBLK / 4 == 4 * NT && TX * TY * RBW == 4 * NT, "four prefetched words per thread");
    static_assert(TX * TY == 2 * NT && kNLCap == 2 * NT, "two segment prefixes and two node links per thread");
    // Block entries, root bitmaps and node counts were final before this grid's predecessor (the
    // scan and link pass) started: that grid waits for the merge to complete before it lets this
    // one launch.  So they are read before the wait -- the entries into registers, the bitmap and
    // count into shared memory (cp.async) -- and the segment prefixes and node links, which the
    // predecessor writes, are copied after it.  With a fixed tile order (no work queue) the next
    // tile's fetches are issued before the current tile's labels are written.
    uint4 nL[4];
    auto fetch = [&](int64_t t) {
#pragma unroll
        for (int i = 0; i < 4; ++i) nL[i] = __ldcg(reinterpret_cast<const uint4 *>(lab + t * NBLK) + tid + i * NT);
        cp_async16(&RB[4 * tid], w.rbits + t * (TX * TY * RBW) + 4 * tid);
        if (tid == NT - 1) cp_async4(&snb, w.nb + t);
        cp_async_commit();
    };
    auto fetch_links = [&](int64_t t) {
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = tid + i * NT;
            cp_async8(&NL[r], w.nlink + t * MAXB + r);
            const int X = r / TY, Y = r % TY;
            if (X < g.nx && Y < g.ny)
                cp_async4(&segb[r], w.segpref + im.seg_base + (int64_t(g.x0 + X) * im.d1 + (g.y0 + Y)) * im.t2 + g.tx2);
        }
        if (tid == 0) cp_async4(&segb[TX * TY], w.segpref + im.seg_base);
        cp_async_commit();
    };
    const bool fixed_order = w.queue == nullptr;
    ItemLoop loop{w.queue ? w.queue + 4 : nullptr, w.n_tiles};
    int64_t t = loop.first(&qslot);
    if (t < w.n_tiles) fetch(t);
    for (bool first = true; t < w.n_tiles; t = loop.next(t, &qslot), first = false) {
        if (!fixed_order && !first) fetch(t);   // a work queue gives the next tile only now
        if (first) grid_dep_wait();   // segment prefixes and node links from here on
        if (first || !fixed_order) fetch_links(t);
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
        const int64_t rs0 = int64_t(im.d1) * im.d2;
#pragma unroll
        for (int i = 0; i < 4; ++i) reinterpret_cast<uint4 *>(Ls)[tid + i * NT] = nL[i];
        cp_async_wait();
        __syncthreads();
        const uint32_t nb = snb, base0 = segb[TX * TY];
        if (t == im.tile_base && tid == 0)
            w.ncomp[im.index] = int64_t(w.segpref[im.seg_base + int64_t(im.d0) * im.d1 * im.t2] - base0);
        for (int b = tid; b < NBLK; b += NT) {
            const uint32_t e = Ls[b];
            if (!(e & ROOT_FLAG)) continue;
            const uint32_t key = e & (ROOT_FLAG - 1);
            const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
            const uint32_t *row = &RB[(X * TY + Y) * RBW];
            uint32_t rank = __popc(row[Z >> 5] & ((1u << (Z & 31)) - 1u));
            for (int k = 0; k < (Z >> 5); ++k) rank += __popc(row[k]);
            LT[b] = 1u + (segb[X * TY + Y] - base0) + rank;
        }
        __syncthreads();
        // Border components linked under another tile's component: the label of that root, its
        // segment's prefix plus its rank among the first voxels left there (both resolved by the
        // link pass).
        for (uint32_t j = tid; j < nb; j += NT) {
            const uint2 e = j < uint32_t(kNLCap) ? NL[j] : __ldcg(w.nlink + t * MAXB + j);
            if (e.x == kNone) continue;
            const uint32_t nr = e.y >> 16;
            if (GUARD(w, nr < uint32_t(NBLK) && e.x < w.n_segs, 402, t * MAXB + j))
                LT[nr] = 1u + (__ldcg(w.segpref + e.x) - base0) + (e.y & 0xFFFFu);
        }
        __syncthreads();
        if (fixed_order && t + gridDim.x < w.n_tiles) {   // RB, NL, segb and snb are free now
            fetch(t + gridDim.x);
            fetch_links(t + gridDim.x);
        }

        // Output: one unit = two blocks along d2 in all four voxel rows (X, Y) they cover: the two
        // entries and labels are looked up once for four 16-byte stores.
        for (int u = tid; u < TB0 * TB1 * (TB2 / 2); u += NT) {
            const int q = u % (TB2 / 2), r = u / (TB2 / 2);
            const int b0 = r / TB1, b1 = r % TB1;
            if (2 * b0 >= g.nx || 2 * b1 >= g.ny || 4 * q >= g.nz) continue;
            const int bb = blk(b0, b1, 2 * q);
            const uint32_t e0 = Ls[bb], e1 = Ls[bb + 1];
            const uint32_t m0 = e0 >> 24, m1 = e1 >> 24;
            if (!GUARD(w, !m0 || (e0 & ROOT_FLAG) || (Ls[(e0 & 0x7FFFFFu) % NBLK] & ROOT_FLAG && (e0 & 0x7FFFFFu) < NBLK), 403, e0)) continue;
            const uint32_t l0 = m0 ? ((e0 & ROOT_FLAG) ? LT[bb] : LT[e0 & 0x7FFFFFu]) : 0u;
            const uint32_t l1 = m1 ? ((e1 & ROOT_FLAG) ? LT[bb + 1] : LT[e1 & 0x7FFFFFu]) : 0u;
            const bool full = 4 * q + 4 <= g.nz;
#pragma unroll
            for (int ij = 0; ij < 4; ++ij) {
                const int X = 2 * b0 + (ij >> 1), Y = 2 * b1 + (ij & 1);
                if (X >= g.nx || Y >= g.ny) continue;
                const int sh = 2 * ij;   // mask bit of voxel (i, j, k) is 4i + 2j + k
                int4 v;
                v.x = ((m0 >> sh) & 1u) ? int(l0) : 0;
                v.y = ((m0 >> (sh + 1)) & 1u) ? int(l0) : 0;
                v.z = ((m1 >> sh) & 1u) ? int(l1) : 0;
                v.w = ((m1 >> (sh + 1)) & 1u) ? int(l1) : 0;
                int32_t *dst = im.out + (g.x0 + X) * rs0 + int64_t(g.y0 + Y) * im.d2 + g.z0 + 4 * q;
                if (full && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                    __stcs(reinterpret_cast<int4 *>(dst), v);
                } else {
                    const int n = min(4, g.nz - 4 * q);
                    dst[0] = v.x;
                    if (n > 1) dst[1] = v.y;
                    if (n > 2) dst[2] = v.z;
                    if (n > 3) dst[3] = v.w;
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace be

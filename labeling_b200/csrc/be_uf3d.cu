// be_uf3d.cu -- 3D Block-Equivalence labeling, union-find form (26-connectivity, 2x2x2 blocks).
//
// Replaces the reference's BLEQ3D_Init / BLEQ3D_Scan / BLEQ3D_Analyze / BLEQ3D_SetFinalLabels
// (LabelingAlgs.cl:740-979) and their host loop (LabelingAlgs.cpp:1443-1536) with the same
// five-launch structure as the 2D pipeline (be_uf2d.cu):
//
//   k_tile_local_3d   one CTA per 16 x 32 x 64-voxel tile (8 x 16 x 32 blocks): 16-byte loads,
//                     8-bit block masks, shared-memory union-find over the 13 preceding
//                     neighbours, flatten, per-component first-voxel key (atomicMin), one uint32
//                     per block, segment root counts, border components exported as nodes.
//   k_merge_3d        global union-find over nodes across the +d0 / +d1 / +d2 tile faces.
//   k_post_3d         ranks of surviving border roots + scan-chunk sums.
//   k_segscan         exclusive scan of the segment counts (be_scan.cu).
//   k_tile_write_3d   resolves canonical labels and writes int32 voxels with 16-byte stores.
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
// Within a tile the union keeps the smaller block index as the root; the component's key (its
// smallest first-voxel index) is then gathered per root with atomicMin.
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
constexpr int ZG = TB2 / 8;                 // 8-block groups along d2
constexpr int ITEMS = TB0 * TB1 * ZG;       // items of 8 blocks
constexpr int RBW = TZ / 32;                // root-bitmap words per voxel row
constexpr uint32_t ROOT_FLAG = 1u << 23;
constexpr int MQ3CAP = NBLK;                // merge-queue capacity (pairs per round)

static_assert(NBLK <= (1 << 13), "tile-local block index must fit the entry payload");
static_assert(TX * TY * TZ <= (1 << 23), "tile-local key must fit the entry payload");
static_assert(ITEMS % NT == 0, "items must divide evenly");
static_assert(NPERIM < 65536 && MAXB < 4096, "border encodings");

// Voxel-offset selector of a block side along one axis: offset 0 (d = -1), 1 (d = +1) or both.
__device__ __forceinline__ uint32_t sel_axis(int axis, int d)
{
    // bit v = 4i + 2j + k; axis 0 -> i, 1 -> j, 2 -> k
    constexpr uint32_t lo[3] = {0x0Fu, 0x33u, 0x55u};
    constexpr uint32_t hi[3] = {0xF0u, 0xCCu, 0xAAu};
    return d < 0 ? lo[axis] : d > 0 ? hi[axis] : 0xFFu;
}

__device__ __forceinline__ uint32_t side_sel(int dx, int dy, int dz)
{
    return sel_axis(0, dx) & sel_axis(1, dy) & sel_axis(2, dz);
}

__device__ __forceinline__ bool bconn(uint32_t ma, uint32_t mb, int dx, int dy, int dz)
{
    return (ma & side_sel(dx, dy, dz)) && (mb & side_sel(-dx, -dy, -dz));
}

__device__ __forceinline__ int blk(int b0, int b1, int b2) { return (b0 * TB1 + b1) * TB2 + b2; }

// Byte-packed mask words: byte k = mask of block k.  nzb gives bit 8k = (byte k != 0);
// rep8 repeats a byte selector in all eight bytes.
__device__ __forceinline__ uint64_t nzb(uint64_t x)
{
    x |= x >> 4;
    x |= x >> 2;
    x |= x >> 1;
    return x & 0x0101010101010101ull;
}
__device__ __forceinline__ uint64_t rep8(uint32_t sel) { return uint64_t(sel) * 0x0101010101010101ull; }

// Out-of-line merge keeps the kernel's code small.
__device__ __noinline__ void merge_blocks3(uint32_t *P, uint32_t a, uint32_t b) { smerge(P, a, b); }

// Tile-local key of the first voxel of a block.
__device__ __forceinline__ uint32_t local_key(int b, uint32_t m)
{
    const int v = __ffs(m) - 1;
    const int b2 = b % TB2, b1 = (b / TB2) % TB1, b0 = b / (TB1 * TB2);
    const int X = 2 * b0 + (v >> 2), Y = 2 * b1 + ((v >> 1) & 1), Z = 2 * b2 + (v & 1);
    return uint32_t((X * TY + Y) * TZ + Z);
}

__device__ __forceinline__ uint32_t nib2byte(uint32_t x)
{
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    return x;
}

// 16 foreground bits along d2 (8 blocks x 2 voxels) -> per block 2-bit field in its byte.
__device__ __forceinline__ uint2 pairs_to_bytes(uint32_t bits16)
{
    const uint32_t n = pairs_to_nibbles(bits16);
    return make_uint2(nib2byte(n), nib2byte(n >> 16));
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
    const int axis = f >> 1, off = f & 1;
    uint32_t r = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const int i = v >> 2, j = (v >> 1) & 1, k = v & 1;
        const int o = axis == 0 ? i : axis == 1 ? j : k;
        if (o != off || !((m >> v) & 1u)) continue;
        const int ta = axis == 0 ? j : i, tb = axis == 2 ? j : k;
        r |= 1u << (ta * 2 + tb);
    }
    return r;
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
    f = 0;
    int q = p;
    while (f < 5 && q >= face_base(f + 1) - face_base(f)) { q -= face_base(f + 1) - face_base(f); ++f; }
    const int axis = f >> 1, hi = f & 1;
    if (axis == 0) { b0 = hi ? g.n0 - 1 : 0; b1 = q / TB2; b2 = q % TB2; }
    else if (axis == 1) { b1 = hi ? g.n1 - 1 : 0; b0 = q / TB2; b2 = q % TB2; }
    else { b2 = hi ? g.n2 - 1 : 0; b0 = q / TB1; b1 = q % TB1; }
    return b0 < g.n0 && b1 < g.n1 && b2 < g.n2;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Tile-local labeling.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(NT, 4) k_tile_local_3d(ImgList3D L, Work w)
{
    __shared__ uint32_t P[NBLK];
    __shared__ uint32_t KQ[NBLK];   // merge queue in Phase B, then first-voxel keys (KM)
    uint32_t *const MQ3 = KQ, *const KM = KQ;
    __shared__ __align__(16) uint8_t M[NBLK];
    __shared__ uint32_t RB[TX * TY * RBW];
    __shared__ uint32_t BF[NBLK / 32];
    __shared__ uint32_t BP[NBLK / 32];
    __shared__ uint32_t tmp[NT / 32 + 1];
    __shared__ uint32_t mqn3[4 * (ITEMS / NT)];      // queue length of each round
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x;
    uint32_t *lab = reinterpret_cast<uint32_t *>(w.lab);
    ItemLoop loop{w.queue ? w.queue + 0 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
        const uint32_t thr4 = uint32_t(im.thr) * 0x01010101u;
        const int64_t rs0 = int64_t(im.d1) * im.d2;   // stride of d0 in voxels

        for (int i = tid; i < TX * TY * RBW; i += NT) RB[i] = 0;
        if (tid < NBLK / 32) BF[tid] = 0;
        if (tid < 4 * (ITEMS / NT)) mqn3[tid] = 0;

        // Phase A: masks and runs along d2.
        uint64_t masks[ITEMS / NT];
#pragma unroll
        for (int it_i = 0; it_i < ITEMS / NT; ++it_i) {
            const int it = tid + it_i * NT;
            const int zg = it % ZG, b1 = (it / ZG) % TB1, b0 = it / (ZG * TB1);
            uint2 acc = make_uint2(0, 0);
            if (b0 < g.n0 && b1 < g.n1 && 16 * zg < g.nz) {
                const int zz = g.z0 + 16 * zg;
                const int n = min(16, g.nz - 16 * zg);
#pragma unroll
                for (int ij = 0; ij < 4; ++ij) {
                    const int i = ij >> 1, j = ij & 1;
                    const int X = g.x0 + 2 * b0 + i, Y = g.y0 + 2 * b1 + j;
                    if (X >= im.d0 || Y >= im.d1) continue;
                    const uint8_t *row = im.in + X * rs0 + int64_t(Y) * im.d2 + zz;
                    uint32_t bits = 0;
                    if (n == 16 && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
                        bits = fg16(__ldg(reinterpret_cast<const uint4 *>(row)), thr4);
                    } else {
                        for (int z = 0; z < n; ++z) bits |= uint32_t(row[z] > im.thr) << z;
                    }
                    const uint2 pb = pairs_to_bytes(bits);
                    const int sh = 4 * i + 2 * j;
                    acc.x |= pb.x << sh;
                    acc.y |= pb.y << sh;
                }
            }
            masks[it_i] = (uint64_t(acc.y) << 32) | acc.x;
            const int bb = blk(b0, b1, 8 * zg);
            *reinterpret_cast<uint2 *>(&M[bb]) = acc;
            uint32_t run = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t m = uint32_t(masks[it_i] >> (8 * k)) & 0xFFu;
                if (!m) continue;
                const uint32_t mp = k ? uint32_t(masks[it_i] >> (8 * (k - 1))) & 0xFFu : 0u;
                if (!(k && bconn(m, mp, 0, 0, -1))) run = bb + k;
                P[bb + k] = run;
            }
        }
        __syncthreads();

        // Phase B: merges with the 13 preceding neighbours inside the tile, decided for the 8
        // blocks of a group at once on byte-packed masks (bit 8k = block k): the 12 neighbours
        // in the four preceding rows (d0-1, d1-1 / d0-1, d1 / d0-1, d1+1 / d0, d1-1) and, at the
        // group's first block, the block before it along d2.  One round per (item, row): every
        // lane queues its links in shared memory, then all lanes merge the queue, so lanes with
        // many links do not hold up their warp.  A round queues at most NT * (3 * 8 + 1) pairs;
        // the queue holds NBLK (it shares its memory with the keys of Phase C), and pairs beyond
        // it are merged in place.
#pragma unroll
        for (int it_i = 0; it_i < ITEMS / NT; ++it_i)
#pragma unroll 1
        for (int row = 0; row < 4; ++row) {
            const int round = 4 * it_i + row;
            const int it = tid + it_i * NT;
            const int zg = it % ZG, b1 = (it / ZG) % TB1, b0 = it / (ZG * TB1);
            const uint64_t ms = masks[it_i];
            const int bb = blk(b0, b1, 8 * zg);
            const int dx = row < 3 ? -1 : 0, dy = row < 3 ? row - 1 : -1;
            const int n0 = b0 + dx, n1 = b1 + dy;
            const int nb0 = (n0 >= 0 && n1 >= 0 && n1 < TB1) ? blk(n0, n1, 8 * zg) : -1;
            uint64_t c[3] = {0, 0, 0};
            bool link_z = false;
            if (ms) {
                const uint64_t ML = zg > 0 ? M[bb - 1] : 0u;
                // hz: block k is joined along d2 to block k-1 (same run)
                const uint64_t hz = nzb(ms & rep8(side_sel(0, 0, -1))) &
                                    nzb(((ms << 8) | ML) & rep8(side_sel(0, 0, 1)));
                link_z = row == 0 && (hz & 1u);
                if (nb0 >= 0) {
                    const uint2 nv = *reinterpret_cast<const uint2 *>(&M[nb0]);
                    const uint64_t N = (uint64_t(nv.y) << 32) | nv.x;
                    const uint64_t NL = zg > 0 ? M[nb0 - 1] : 0u;
                    const uint64_t NR = 8 * zg + 8 < TB2 ? M[nb0 + 8] : 0u;
                    if (N | NL | NR) {
#pragma unroll
                        for (int dz = -1; dz <= 1; ++dz) {
                            const uint64_t Ns = dz < 0 ? (N << 8) | NL : dz > 0 ? (N >> 8) | (NR << 56) : N;
                            c[dz + 1] = nzb(ms & rep8(side_sel(dx, dy, dz))) &
                                        nzb(Ns & rep8(side_sel(-dx, -dy, -dz)));
                        }
                        // Skip rules (as in the 2D kernel: every chain of reasons runs toward
                        // smaller d2 along the run and ends at a link that is made).
                        // (1) The previous block of the run touches the same block of row N.
                        const uint64_t raw1 = c[1];
                        c[0] &= ~(hz & (raw1 << 8));
                        c[1] &= ~(hz & (c[2] << 8));
                        // (2) Blocks of row N joined along d2 to the block this one touches
                        //     with dz = 0.
                        const uint64_t hzN = nzb(N & rep8(side_sel(0, 0, -1))) &
                                             nzb(((N << 8) | NL) & rep8(side_sel(0, 0, 1)));
                        const uint64_t hzN1 =
                            (hzN >> 8) |
                            (uint64_t((NR & side_sel(0, 0, -1)) && ((N >> 56) & side_sel(0, 0, 1))) << 56);
                        c[0] &= ~(raw1 & hzN);
                        c[2] &= ~(raw1 & hzN1);
                    }
                }
            }
            const uint32_t n = __popcll(c[0]) + __popcll(c[1]) + __popcll(c[2]) + (link_z ? 1u : 0u);
            uint32_t pos = warp_reserve(&mqn3[round], n);
            auto push = [&](uint32_t x, uint32_t y) {
                if (pos < uint32_t(MQ3CAP)) MQ3[pos] = (x << 16) | y;
                else smerge(P, x, y);   // queue full: merge in place
                ++pos;
            };
            if (link_z) push(uint32_t(bb), uint32_t(bb - 1));
            uint64_t todo = c[0] | c[1] | c[2];
            while (todo) {
                const int k = (__ffsll(todo) - 1) >> 3;
                const uint64_t bit = uint64_t(1) << (8 * k);
                todo &= ~bit;
                if (c[0] & bit) push(uint32_t(bb + k), uint32_t(nb0 + k - 1));
                if (c[1] & bit) push(uint32_t(bb + k), uint32_t(nb0 + k));
                if (c[2] & bit) push(uint32_t(bb + k), uint32_t(nb0 + k + 1));
            }
            __syncthreads();
            const uint32_t nq = min(mqn3[round], uint32_t(MQ3CAP));
            for (uint32_t q = tid; q < nq; q += NT) smerge(P, MQ3[q] >> 16, MQ3[q] & 0xFFFFu);
            __syncthreads();
        }

        // Phase C: roots (read-only finds: all merges are done) and per-component first-voxel
        // key.  Each root first stores its own block's key; a block of the component then needs
        // the atomic only when its key is smaller, which keeps the atomics off the (common) case
        // of a large component whose blocks all follow its root block.
        uint16_t roots[ITEMS / NT][8];
#pragma unroll
        for (int it_i = 0; it_i < ITEMS / NT; ++it_i) {
            const int it = tid + it_i * NT;
            const int zg = it % ZG, b1 = (it / ZG) % TB1, b0 = it / (ZG * TB1);
            const uint64_t ms = masks[it_i];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t m = uint32_t(ms >> (8 * k)) & 0xFFu;
                if (!m) continue;
                const int b = blk(b0, b1, 8 * zg + k);
                const uint32_t root = sflatten(P, b);
                roots[it_i][k] = uint16_t(root);
                if (root == uint32_t(b)) KM[b] = local_key(b, m);
            }
        }
        __syncthreads();
#pragma unroll
        for (int it_i = 0; it_i < ITEMS / NT; ++it_i) {
            const int it = tid + it_i * NT;
            const int zg = it % ZG, b1 = (it / ZG) % TB1, b0 = it / (ZG * TB1);
            const uint64_t ms = masks[it_i];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t m = uint32_t(ms >> (8 * k)) & 0xFFu;
                if (!m) continue;
                const int b = blk(b0, b1, 8 * zg + k);
                const uint32_t root = roots[it_i][k];
                if (root == uint32_t(b)) continue;
                const uint32_t key = local_key(b, m);
                if (key < KM[root]) atomicMin(&KM[root], key);
            }
        }
        __syncthreads();
#pragma unroll
        for (int it_i = 0; it_i < ITEMS / NT; ++it_i) {
            const int it = tid + it_i * NT;
            const int zg = it % ZG, b1 = (it / ZG) % TB1, b0 = it / (ZG * TB1);
            const uint64_t ms = masks[it_i];
            const int bb = blk(b0, b1, 8 * zg);
            uint32_t e[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t m = uint32_t(ms >> (8 * k)) & 0xFFu;
                e[k] = 0;
                if (!m) continue;
                const int b = bb + k;
                const uint32_t root = roots[it_i][k];
                if (root == uint32_t(b)) {
                    const uint32_t key = KM[b];
                    e[k] = (m << 24) | ROOT_FLAG | key;
                    const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
                    if (GUARD(w, key < uint32_t(TX * TY * TZ), 101, key))
                        atomicOr(&RB[(X * TY + Y) * RBW + (Z >> 5)], 1u << (Z & 31));
                } else {
                    e[k] = (m << 24) | root;
                }
            }
            uint4 *dst = reinterpret_cast<uint4 *>(lab + t * NBLK + bb);
            dst[0] = make_uint4(e[0], e[1], e[2], e[3]);
            dst[1] = make_uint4(e[4], e[5], e[6], e[7]);
        }
        __syncthreads();

        // Phase D: segment counts and border nodes.
        for (int r = tid; r < TX * TY; r += NT) {
            const int X = r / TY, Y = r % TY;
            if (X >= g.nx || Y >= g.ny) continue;
            uint32_t cnt = 0;
#pragma unroll
            for (int k = 0; k < RBW; ++k) cnt += __popc(RB[r * RBW + k]);
            const int64_t si = im.seg_base + (int64_t(g.x0 + X) * im.d1 + (g.y0 + Y)) * im.t2 + g.tx2;
            if (GUARD(w, si >= 0 && si < w.n_segs, 104, si)) w.segcnt[si] = uint8_t(cnt);
        }
        for (int p = tid; p < NPERIM; p += NT) {
            int f, b0, b1, b2;
            if (!perim_pos3(p, g, f, b0, b1, b2)) continue;
            const int b = blk(b0, b1, b2);
            if (!M[b]) continue;
            const uint32_t rb = sfind_ro(P, b);
            atomicOr(&BF[rb >> 5], 1u << (rb & 31));
        }
        __syncthreads();
        uint32_t nb;
        const uint32_t pre = block_exscan<NT>(tid < NBLK / 32 ? __popc(BF[tid]) : 0u, tmp, &nb);
        if (tid < NBLK / 32) BP[tid] = pre;
        __syncthreads();
        if (tid < NBLK / 32) {
            uint32_t bits = BF[tid];
            uint32_t j = pre;
            while (bits) {
                const int bit = __ffs(bits) - 1;
                bits &= bits - 1;
                const uint32_t rb = tid * 32 + bit;
                const uint32_t key = KM[rb];
                if (!GUARD(w, key < uint32_t(TX * TY * TZ) && j < uint32_t(MAXB), 102, (uint64_t(j) << 32) | key))
                    break;
                const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
                const uint32_t *row = &RB[(X * TY + Y) * RBW];
                uint32_t rank = __popc(row[Z >> 5] & ((1u << (Z & 31)) - 1u));
                for (int k = 0; k < (Z >> 5); ++k) rank += __popc(row[k]);
                const int64_t node = t * MAXB + j;
                w.nroot[node] = uint16_t(rb);
                w.nkey[node] = uint32_t((int64_t(g.x0 + X) * im.d1 + (g.y0 + Y)) * im.d2 + (g.z0 + Z));
                w.nlrank[node] = uint16_t(rank);
                w.gp[node] = uint32_t(node);
                ++j;
            }
        }
        for (int p = tid; p < NPERIM; p += NT) {
            int f, b0, b1, b2;
            uint16_t ent = 0;
            if (perim_pos3(p, g, f, b0, b1, b2)) {
                const int b = blk(b0, b1, b2);
                const uint32_t m = M[b];
                if (m) {
                    const uint32_t rb = sfind_ro(P, b);
                    const uint32_t j = BP[rb >> 5] + __popc(BF[rb >> 5] & ((1u << (rb & 31)) - 1u));
                    ent = uint16_t((j << 4) | face_bits(m, f));
                }
            }
            w.perim[t * NPERIM + p] = ent;
        }
        if (tid == 0) w.nb[t] = nb;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Cross-tile merge over the +d0, +d1 and +d2 faces.
// ---------------------------------------------------------------------------------------------
namespace {

__device__ void gunion3d(const Img3D &im, Work &w, uint32_t a, uint32_t b)
{
    for (;;) {
        a = gfind(w.gp, a);
        b = gfind(w.gp, b);
        if (a == b) return;
        uint32_t ka = w.nkey[a], kb = w.nkey[b];
        if (ka < kb) {
            uint32_t t = a; a = b; b = t;
            t = ka; ka = kb; kb = t;
        }
        if (atomicCAS(&w.gp[a], a, b) == a) {
            const int64_t row = ka / uint32_t(im.d2), z = ka - row * im.d2;
            dec_u8(w.segcnt, im.seg_base + row * im.t2 + z / TZ);
            return;
        }
    }
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
constexpr int kGQ3 = 1024;   // queued global unions per tile (more are done at once)
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

__global__ void __launch_bounds__(kT3MergeThreads, 4) k_merge_3d(ImgList3D L, Work w)
{
    __shared__ uint32_t qslot;
    __shared__ uint32_t lp[MAXB + NPF];   // local union-find: this tile's nodes, then staged positions
    __shared__ uint32_t nbid[NPF];        // global node id across the face, kNone = none
    __shared__ uint8_t nbf[NPF];          // its face bits
    __shared__ uint2 gq[kGQ3];
    __shared__ uint32_t nq;
    ItemLoop loop{w.queue ? w.queue + 1 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
        for (int i = threadIdx.x; i < MAXB + NPF; i += kT3MergeThreads) lp[i] = uint32_t(i);
        if (threadIdx.x == 0) nq = 0;
        for (int e = threadIdx.x; e < PF0; e += kT3MergeThreads) stage_face<0>(im, g, w, e, nbid, nbf);
        for (int e = threadIdx.x; e < PF1; e += kT3MergeThreads) stage_face<1>(im, g, w, e, nbid, nbf);
        for (int e = threadIdx.x; e < PF2; e += kT3MergeThreads) stage_face<2>(im, g, w, e, nbid, nbf);
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
        // Pairs: a pair whose two elements are already one local set is implied by pairs queued
        // before it (smerge_joined); the rest are unioned globally after the loop.
        for (int p = threadIdx.x; p < NPLUS; p += kT3MergeThreads) {
            int u = 0, v = 0, ebase, pitch;
            uint32_t A;
            if (p < FaceAx<0>::NPOS) {
                A = plus_entry<0>(im, g, w, t, p, u, v);
                ebase = FaceAx<0>::EBASE; pitch = FaceAx<0>::PITCH;
            } else if (p < FaceAx<0>::NPOS + FaceAx<1>::NPOS) {
                A = plus_entry<1>(im, g, w, t, p - FaceAx<1>::PBASE, u, v);
                ebase = FaceAx<1>::EBASE; pitch = FaceAx<1>::PITCH;
            } else {
                A = plus_entry<2>(im, g, w, t, p - FaceAx<2>::PBASE, u, v);
                ebase = FaceAx<2>::EBASE; pitch = FaceAx<2>::PITCH;
            }
            if (!A || !GUARD(w, (A >> 4) < w.nb[t] && (A >> 4) < uint32_t(MAXB), 204, (uint64_t(t) << 16) | (A >> 4)))
                continue;
            const uint32_t fa = A & 15u, ja = A >> 4, nA = uint32_t(t * MAXB + ja);
#pragma unroll
            for (int da = -1; da <= 1; ++da) {
#pragma unroll
                for (int db = -1; db <= 1; ++db) {
                    if (!(fa & face_sel(da, db))) continue;
                    const int e = ebase + (u + 1 + da) * pitch + (v + 1 + db);
                    const uint32_t id = nbid[e];
                    if (id == kNone || !(nbf[e] & face_sel(-da, -db))) continue;
                    if (!smerge_joined(lp, ja, uint32_t(MAXB + e))) continue;
                    const uint32_t slot = atomicAdd(&nq, 1u);
                    if (slot < uint32_t(kGQ3)) gq[slot] = make_uint2(nA, id);
                    else gunion3d(im, w, nA, id);
                }
            }
        }
        __syncthreads();
        const uint32_t nqt = min(nq, uint32_t(kGQ3));
        for (uint32_t i = threadIdx.x; i < nqt; i += kT3MergeThreads) gunion3d(im, w, gq[i].x, gq[i].y);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Post-merge ranks of surviving border roots, and scan-chunk sums.
// ---------------------------------------------------------------------------------------------
namespace {

__device__ void post_tile_3d(const ImgList3D &L, Work &w, int64_t t)
{
    __shared__ uint32_t LB[TX * TY * RBW];   // keys of linked nodes
    const Img3D im = L.get(t);
    const TileGeo g = tile_geo(im, t);
    const uint32_t nb = w.nb[t];
    for (int i = threadIdx.x; i < TX * TY * RBW; i += blockDim.x) LB[i] = 0;
    __syncthreads();
    auto local = [&](uint32_t key, int &X, int &Y, int &Z) {
        const uint32_t row = key / uint32_t(im.d2);
        Z = int(key - row * uint32_t(im.d2)) - g.z0;
        const uint32_t xg = row / uint32_t(im.d1);
        Y = int(row - xg * uint32_t(im.d1)) - g.y0;
        X = int(xg) - g.x0;
    };
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const int64_t node = t * MAXB + j;
        if (w.gp[node] == uint32_t(node)) continue;
        int X, Y, Z;
        local(w.nkey[node], X, Y, Z);
        if (GUARD(w, X >= 0 && X < TX && Y >= 0 && Y < TY && Z >= 0 && Z < TZ, 301, w.nkey[node]))
            atomicOr(&LB[(X * TY + Y) * RBW + (Z >> 5)], 1u << (Z & 31));
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const int64_t node = t * MAXB + j;
        if (w.gp[node] != uint32_t(node)) continue;
        int X, Y, Z;
        local(w.nkey[node], X, Y, Z);
        if (!GUARD(w, X >= 0 && X < TX && Y >= 0 && Y < TY && Z >= 0 && Z < TZ, 302, w.nkey[node])) continue;
        const uint32_t *row = &LB[(X * TY + Y) * RBW];
        uint32_t cnt = __popc(row[Z >> 5] & ((1u << (Z & 31)) - 1u));
        for (int k = 0; k < (Z >> 5); ++k) cnt += __popc(row[k]);
        w.grank[node] = w.nlrank[node] - cnt;
    }
    __syncthreads();
}

}  // namespace

__global__ void __launch_bounds__(kPostThreads) k_post_3d(ImgList3D L, Work w)
{
    __shared__ uint32_t tmp[kPostThreads / 32 + 1];
    __shared__ uint32_t qslot;
    const int64_t n = w.n_tiles + w.n_chunks;
    ItemLoop loop{w.queue ? w.queue + 2 : nullptr, n};
    for (int64_t it = loop.first(&qslot); it < n; it = loop.next(it, &qslot)) {
        if (it < w.n_tiles) post_tile_3d(L, w, it);
        else chunk_sum<kPostThreads>(w, it - w.n_tiles, tmp);
    }
}

// ---------------------------------------------------------------------------------------------
// Label resolve and write.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_tile_write_3d(ImgList3D L, Work w)
{
    __shared__ __align__(16) uint32_t Ls[NBLK];
    __shared__ uint32_t LT[NBLK];
    __shared__ uint32_t RB[TX * TY * RBW];
    __shared__ uint32_t segb[TX * TY];
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x;
    const uint32_t *lab = reinterpret_cast<const uint32_t *>(w.lab);
    ItemLoop loop{w.queue ? w.queue + 4 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img3D im = L.get(t);
        const TileGeo g = tile_geo(im, t);
        const uint32_t base0 = w.segpref[im.seg_base];
        const int64_t rs0 = int64_t(im.d1) * im.d2;

        for (int i = tid; i < NBLK / 4; i += NT)
            reinterpret_cast<uint4 *>(Ls)[i] = reinterpret_cast<const uint4 *>(lab + t * NBLK)[i];
        for (int i = tid; i < TX * TY * RBW; i += NT) RB[i] = 0;
        for (int r = tid; r < TX * TY; r += NT) {
            const int X = r / TY, Y = r % TY;
            if (X < g.nx && Y < g.ny)
                segb[r] = w.segpref[im.seg_base + (int64_t(g.x0 + X) * im.d1 + (g.y0 + Y)) * im.t2 + g.tx2] - base0;
        }
        if (t == im.tile_base && tid == 0)
            w.ncomp[im.index] = int64_t(w.segpref[im.seg_base + int64_t(im.d0) * im.d1 * im.t2] - base0);
        __syncthreads();

        for (int b = tid; b < NBLK; b += NT) {
            const uint32_t e = Ls[b];
            if (!(e & ROOT_FLAG)) continue;
            const uint32_t key = e & (ROOT_FLAG - 1);
            const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
            if (GUARD(w, key < uint32_t(TX * TY * TZ), 401, key))
                atomicOr(&RB[(X * TY + Y) * RBW + (Z >> 5)], 1u << (Z & 31));
        }
        __syncthreads();
        const uint32_t nb = w.nb[t];
        for (uint32_t j = tid; j < nb; j += NT) {
            const int64_t node = t * MAXB + j;
            if (w.gp[node] == uint32_t(node)) continue;
            if (!GUARD(w, w.nroot[node] < NBLK && (Ls[w.nroot[node] % NBLK] & ROOT_FLAG), 402, node)) continue;
            const uint32_t key = Ls[w.nroot[node]] & (ROOT_FLAG - 1);
            const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
            atomicAnd(&RB[(X * TY + Y) * RBW + (Z >> 5)], ~(1u << (Z & 31)));
        }
        __syncthreads();
        for (int b = tid; b < NBLK; b += NT) {
            const uint32_t e = Ls[b];
            if (!(e & ROOT_FLAG)) continue;
            const uint32_t key = e & (ROOT_FLAG - 1);
            const int Z = key % TZ, Y = (key / TZ) % TY, X = key / (TZ * TY);
            const uint32_t *row = &RB[(X * TY + Y) * RBW];
            uint32_t rank = __popc(row[Z >> 5] & ((1u << (Z & 31)) - 1u));
            for (int k = 0; k < (Z >> 5); ++k) rank += __popc(row[k]);
            LT[b] = 1u + segb[X * TY + Y] + rank;
        }
        __syncthreads();
        for (uint32_t j = tid; j < nb; j += NT) {
            const int64_t node = t * MAXB + j;
            if (w.gp[node] == uint32_t(node)) continue;
            const uint32_t gn = gfind_ro(w.gp, uint32_t(node));
            const uint32_t kg = w.nkey[gn];
            const int64_t row = kg / uint32_t(im.d2), z = kg - row * im.d2;
            const int64_t si = im.seg_base + row * im.t2 + z / TZ;
            if (!GUARD(w, si >= 0 && si <= w.n_segs, 404, si)) continue;
            const uint32_t sb = w.segpref[si] - base0;
            LT[w.nroot[node]] = 1u + sb + w.grank[gn];
        }
        __syncthreads();

        // Output: units of 4 voxels along d2 (2 blocks).
        for (int u = tid; u < TX * TY * (TZ / 4); u += NT) {
            const int q = u % (TZ / 4), r = u / (TZ / 4);
            const int X = r / TY, Y = r % TY;
            if (X >= g.nx || Y >= g.ny || 4 * q >= g.nz) continue;
            const int bb = blk(X >> 1, Y >> 1, 2 * q);
            const uint32_t e0 = Ls[bb], e1 = (2 * q + 1 < TB2) ? Ls[bb + 1] : 0u;
            const uint32_t m0 = e0 >> 24, m1 = e1 >> 24;
            if (!GUARD(w, !m0 || (e0 & ROOT_FLAG) || (Ls[(e0 & 0x7FFFFFu) % NBLK] & ROOT_FLAG && (e0 & 0x7FFFFFu) < NBLK), 403, e0)) continue;
            const uint32_t l0 = m0 ? ((e0 & ROOT_FLAG) ? LT[bb] : LT[e0 & 0x7FFFFFu]) : 0u;
            const uint32_t l1 = m1 ? ((e1 & ROOT_FLAG) ? LT[bb + 1] : LT[e1 & 0x7FFFFFu]) : 0u;
            const int sh = 4 * (X & 1) + 2 * (Y & 1);
            int4 v;
            v.x = ((m0 >> sh) & 1u) ? int(l0) : 0;
            v.y = ((m0 >> (sh + 1)) & 1u) ? int(l0) : 0;
            v.z = ((m1 >> sh) & 1u) ? int(l1) : 0;
            v.w = ((m1 >> (sh + 1)) & 1u) ? int(l1) : 0;
            int32_t *dst = im.out + (g.x0 + X) * rs0 + int64_t(g.y0 + Y) * im.d2 + g.z0 + 4 * q;
            if (4 * q + 4 <= g.nz && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                __stcs(reinterpret_cast<int4 *>(dst), v);
            } else {
                const int n = min(4, g.nz - 4 * q);
                dst[0] = v.x;
                if (n > 1) dst[1] = v.y;
                if (n > 2) dst[2] = v.z;
                if (n > 3) dst[3] = v.w;
            }
        }
        __syncthreads();
    }
}

}  // namespace be

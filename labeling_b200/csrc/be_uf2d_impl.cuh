// be_uf2d_impl.cuh -- the 2D union-find pipeline for one tile shape.  Included by be_uf2d.cu
// once per supported shape, inside a namespace that defines `TBW` and `TBH` (tile width and
// height in 2x2 blocks, TBW * TBH <= 4096, TBW a power of two in [64, 256]).
namespace {

constexpr int TW = 2 * TBW, TH = 2 * TBH;          // tile in pixels
constexpr int NBLK = TBW * TBH;                    // blocks per tile (4096)
constexpr int NPERIM = 2 * (TBW + TBH);            // border positions per tile
constexpr int MAXB = NPERIM;                       // nodes per tile
constexpr int K1_NT = 256;
constexpr int ITEMS = NBLK / 8;                    // 8-block row groups per tile
constexpr int GROUPS = TBW / 8;                    // groups per block row
constexpr int MQCAP = 2048;                        // merge-queue capacity (pairs per tile)

static_assert(NBLK <= 4096, "tile-local block index must fit 12 bits");
static_assert(MAXB < 4096, "node index must fit 12 bits");

// Mask bits: 0 = top-left, 1 = top-right, 2 = bottom-left, 3 = bottom-right pixel.
__device__ __forceinline__ uint32_t slot_of(int r, int c, uint32_t m)
{
    return uint32_t(r) * (2 * TBW) + ((m & 3u) ? 0u : uint32_t(TBW)) + uint32_t(c);
}

// Pixel offset (row, column) of a block's first foreground pixel, inside the block.
__device__ __forceinline__ void first_px(uint32_t m, int &dy, int &dx)
{
    if (m & 3u) { dy = 0; dx = (m & 1u) ? 0 : 1; }
    else { dy = 1; dx = (m & 4u) ? 0 : 1; }
}

__device__ __forceinline__ bool hconn(uint32_t left, uint32_t right)
{
    return (left & 0xAu) && (right & 0x5u);
}

// Block position of border position p of a tile with nbr x nbc valid blocks.
__device__ __forceinline__ bool perim_pos(int p, int nbr, int nbc, int &r, int &c)
{
    if (p < TBW) { r = 0; c = p; return c < nbc; }
    if (p < 2 * TBW) { r = nbr - 1; c = p - TBW; return c < nbc; }
    if (p < 2 * TBW + TBH) { r = p - 2 * TBW; c = 0; return r < nbr; }
    r = p - 2 * TBW - TBH; c = nbc - 1;
    return r < nbr;
}

// Nibble-packed mask words: nibble k = mask of block k; nb_bN gives bit N of every nibble at
// bit 4k, so block-wise predicates of 8 blocks are a few bitwise operations.
__device__ __forceinline__ uint32_t nb_b0(uint32_t x) { return x & 0x11111111u; }
__device__ __forceinline__ uint32_t nb_b1(uint32_t x) { return (x >> 1) & 0x11111111u; }
__device__ __forceinline__ uint32_t nb_b2(uint32_t x) { return (x >> 2) & 0x11111111u; }
__device__ __forceinline__ uint32_t nb_b3(uint32_t x) { return (x >> 3) & 0x11111111u; }
__device__ __forceinline__ uint32_t nb_lft(uint32_t x) { return nb_b0(x) | nb_b2(x); }
__device__ __forceinline__ uint32_t nb_rgt(uint32_t x) { return nb_b1(x) | nb_b3(x); }

// Four bytes (each < 16) -> four nibbles.
__device__ __forceinline__ uint32_t bytes_to_nibbles(uint32_t x)
{
    x = (x | (x >> 4)) & 0x00FF00FFu;
    return (x | (x >> 8)) & 0xFFFFu;
}

__device__ __forceinline__ uint32_t nib2byte(uint32_t x)
{
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    return x;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Tile-local labeling.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(K1_NT, 4) k_tile_local_2d(ImgList2D L, Work w)
{
    __shared__ uint32_t P[2 * NBLK];
    __shared__ __align__(16) uint8_t M[NBLK];
    __shared__ uint32_t RB[TH][TW / 32];
    __shared__ uint32_t BF[NBLK / 32];
    __shared__ uint32_t BP[NBLK / 32];
    __shared__ uint32_t MQ[MQCAP];          // merge queue: (slot_a << 16) | slot_b
    __shared__ uint32_t mqn[2];
    __shared__ uint32_t tmp[K1_NT / 32 + 1];
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x;
    uint16_t *lab = reinterpret_cast<uint16_t *>(w.lab);
    ItemLoop loop{w.queue ? w.queue + 0 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img2D im = L.get(t);
        const int64_t lt = t - im.tile_base;
        const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
        const int y0 = ty * TH, x0 = tx * TW;
        const int nrp = min(TH, im.rows - y0), ncp = min(TW, im.cols - x0);
        const int nbr = (nrp + 1) >> 1, nbc = (ncp + 1) >> 1;
        const uint32_t thr4 = uint32_t(im.thr) * 0x01010101u;

        for (int i = tid; i < TH * (TW / 32); i += K1_NT) (&RB[0][0])[i] = 0;
        if (tid < NBLK / 32) BF[tid] = 0;
        if (tid < 2) mqn[tid] = 0;

        // Phase A: load pixels, build block masks, seed the union-find with horizontal runs.
        uint32_t masks[ITEMS / K1_NT];
#pragma unroll
        for (int i = 0; i < ITEMS / K1_NT; ++i) {
            const int it = tid + i * K1_NT, r = it / GROUPS, g = it % GROUPS;
            uint32_t top = 0, bot = 0;
            if (r < nbr && 16 * g < ncp) {
                const int py = y0 + 2 * r, px = x0 + 16 * g;
                const uint8_t *row0 = im.in + int64_t(py) * im.in_pitch + px;
                const bool row1 = py + 1 < im.rows;
                const bool vec = (16 * g + 16 <= ncp) &&
                                 ((reinterpret_cast<uintptr_t>(row0) | uintptr_t(im.in_pitch)) & 15) == 0;
                if (vec) {
                    top = fg16(__ldg(reinterpret_cast<const uint4 *>(row0)), thr4);
                    if (row1) bot = fg16(__ldg(reinterpret_cast<const uint4 *>(row0 + im.in_pitch)), thr4);
                } else {
                    const int n = min(16, ncp - 16 * g);
                    for (int x = 0; x < n; ++x) {
                        top |= uint32_t(row0[x] > im.thr) << x;
                        if (row1) bot |= uint32_t(row0[im.in_pitch + x] > im.thr) << x;
                    }
                }
            }
            const uint32_t ms = pairs_to_nibbles(top) | (pairs_to_nibbles(bot) << 2);
            masks[i] = ms;
            *reinterpret_cast<uint2 *>(&M[r * TBW + 8 * g]) = make_uint2(nib2byte(ms), nib2byte(ms >> 16));
            // Horizontal runs: every block points at its run's smallest slot.  Within the group
            // a prefix minimum finds each run part's minimum; runs that cross group borders are
            // joined with segmented minimum scans over the 16 groups of the block row (one
            // half-warp), so no merge is needed for horizontal links.
            uint32_t pm[8];
            bool inf[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t m = (ms >> (4 * k)) & 15u;
                const uint32_t s = slot_of(r, 8 * g + k, m);
                const bool hc = k > 0 && hconn((ms >> (4 * (k - 1))) & 15u, m);
                pm[k] = hc ? min(pm[k - 1], s) : s;
                inf[k] = k == 0 ? (m != 0) : (inf[k - 1] && hc);
            }
            const uint32_t m0 = ms & 15u, m7 = ms >> 28;
            const uint32_t prev_ms = __shfl_up_sync(0xFFFFFFFFu, ms, 1, GROUPS);
            const bool linkL = g > 0 && hconn(prev_ms >> 28, m0);
            const bool linkR = __shfl_down_sync(0xFFFFFFFFu, uint32_t(linkL), 1, GROUPS) && g + 1 < GROUPS;
            const bool single = inf[7];
            // first_min: minimum of the run part holding block 0 (found by the backward pass).
            uint32_t run = kNone, first_min = kNone;
            uint32_t part[8];
#pragma unroll
            for (int k = 7; k >= 0; --k) {
                const uint32_t m = (ms >> (4 * k)) & 15u;
                const bool last = (k == 7) || !hconn(m, (ms >> (4 * (k + 1))) & 15u);
                if (last) run = pm[k];
                part[k] = run;
            }
            first_min = m0 ? part[0] : kNone;
            const uint32_t last_min = m7 ? pm[7] : kNone;
            // Left-to-right: minimum of the run entering from the left.
            uint32_t fv = last_min;
            uint32_t ff = !(single && linkL);
#pragma unroll
            for (int o = 1; o < GROUPS; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, fv, o, GROUPS);
                const uint32_t f = __shfl_up_sync(0xFFFFFFFFu, ff, o, GROUPS);
                if (g >= o && !ff) { fv = min(fv, v); ff |= f; }
            }
            const uint32_t fprev = __shfl_up_sync(0xFFFFFFFFu, fv, 1, GROUPS);
            const uint32_t fromL = linkL ? fprev : kNone;
            // Right-to-left: minimum of the run leaving to the right.
            uint32_t bv = first_min;
            uint32_t bf = !(single && linkR);
#pragma unroll
            for (int o = 1; o < GROUPS; o <<= 1) {
                const uint32_t v = __shfl_down_sync(0xFFFFFFFFu, bv, o, GROUPS);
                const uint32_t f = __shfl_down_sync(0xFFFFFFFFu, bf, o, GROUPS);
                if (g + o < GROUPS && !bf) { bv = min(bv, v); bf |= f; }
            }
            const uint32_t bnext = __shfl_down_sync(0xFFFFFFFFu, bv, 1, GROUPS);
            const uint32_t fromR = linkR ? bnext : kNone;
            bool inl = m7 != 0;
#pragma unroll
            for (int k = 7; k >= 0; --k) {
                const uint32_t m = (ms >> (4 * k)) & 15u;
                if (k < 7) inl = inl && hconn(m, (ms >> (4 * (k + 1))) & 15u);
                if (!m) continue;
                uint32_t v = part[k];
                if (inf[k]) v = min(v, fromL);
                if (inl) v = min(v, fromR);
                P[slot_of(r, 8 * g + k, m)] = v;
            }
        }
        __syncthreads();

        // Phase B: the links to the row above, decided for the 8 blocks of a group at once on
        // nibble-packed masks (bit 4k = block k), are queued in shared memory and then merged
        // with every lane busy (one round per item, so the queue rarely overflows).
#pragma unroll
        for (int i = 0; i < ITEMS / K1_NT; ++i) {
            const int it = tid + i * K1_NT, r = it / GROUPS, g = it % GROUPS;
            const uint32_t ms = masks[i];
            const int c0 = 8 * g;
            uint32_t *qn = &mqn[i];
            uint32_t hcl = 0, cN = 0, cNW = 0, cNE = 0, U = 0, UL = 0, UR = 0, ML = 0;
            if (ms) {
                ML = c0 > 0 ? M[r * TBW + c0 - 1] : 0u;
                hcl = nb_lft(ms) & ((nb_rgt(ms) << 4) | nb_rgt(ML));
                if (r > 0) {
                    const uint8_t *Urow = &M[(r - 1) * TBW];
                    const uint2 ub = *reinterpret_cast<const uint2 *>(Urow + c0);
                    U = bytes_to_nibbles(ub.x) | (bytes_to_nibbles(ub.y) << 16);
                    UL = c0 > 0 ? Urow[c0 - 1] : 0u;
                    UR = c0 + 8 < TBW ? Urow[c0 + 8] : 0u;
                    const uint32_t top = nb_b0(ms) | nb_b1(ms);
                    const uint32_t uBL = nb_b2(U), uBR = nb_b3(U), uB = uBL | uBR;
                    const uint32_t rawN = top & uB;
                    cN = rawN;
                    cNW = nb_b0(ms) & ((uBR << 4) | nb_b3(UL));
                    cNE = nb_b1(ms) & ((uBL >> 4) | (nb_b2(UR) << 28));
                    // Skip rules.  A link may be skipped when its two blocks are already joined
                    // through links that are made or are themselves skipped for a reason further
                    // left; every chain of reasons runs leftward along the run and ends at a
                    // link that is made.
                    // (1) The left block of the same run touches the same upper block.
                    const uint32_t leftN = ((top << 4) | nb_b0(ML) | nb_b1(ML)) & ((uB << 4) | nb_b2(UL) | nb_b3(UL));
                    const uint32_t leftNE = ((nb_b1(ms) << 4) | nb_b1(ML)) & uBL;
                    cNW &= ~(hcl & leftN);
                    cN &= ~(hcl & leftNE);
                    // (2) The upper diagonal block is joined horizontally to the block straight
                    //     above, which this block touches.
                    const uint32_t uL = nb_lft(U), uR = nb_rgt(U);
                    cNW &= ~(rawN & (((uR << 4) | nb_rgt(UL)) & uL));
                    cNE &= ~(rawN & (uR & ((uL >> 4) | (nb_lft(UR) << 28))));
                }
            }
            const uint32_t n = __popc(cN) + __popc(cNW) + __popc(cNE);
            uint32_t pos = warp_reserve(qn, n);
            auto push = [&](uint32_t a, uint32_t b) {
                if (pos < MQCAP) MQ[pos] = (a << 16) | b;
                else smerge(P, a, b);   // queue full: merge in place
                ++pos;
            };
            uint32_t todo = cN | cNW | cNE;
            while (todo) {
                const int k = (__ffs(todo) - 1) >> 2;
                const uint32_t bit = 1u << (4 * k);
                todo &= ~bit;
                const int c = c0 + k;
                const uint32_t sl = slot_of(r, c, (ms >> (4 * k)) & 15u);
                if (cN & bit) push(sl, slot_of(r - 1, c, (U >> (4 * k)) & 15u));
                if (cNW & bit) push(sl, slot_of(r - 1, c - 1, k ? (U >> (4 * k - 4)) & 15u : UL));
                if (cNE & bit) push(sl, slot_of(r - 1, c + 1, k < 7 ? (U >> (4 * k + 4)) & 15u : UR));
            }
            __syncthreads();
            const uint32_t nq = min(*qn, uint32_t(MQCAP));
            for (uint32_t q = tid; q < nq; q += K1_NT) smerge(P, MQ[q] >> 16, MQ[q] & 0xFFFFu);
            __syncthreads();
        }

        // Phase C: resolve each block's root (read-only: all merges are done), write tile-local
        // labels, mark roots.
#pragma unroll
        for (int i = 0; i < ITEMS / K1_NT; ++i) {
            const int it = tid + i * K1_NT, r = it / GROUPS, g = it % GROUPS;
            const uint32_t ms = masks[i];
            uint32_t e[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t m = (ms >> (4 * k)) & 15u;
                e[k] = 0;
                if (!m) continue;
                const int c = 8 * g + k;
                const uint32_t s = slot_of(r, c, m);
                const uint32_t root = sflatten(P, s);
                const uint32_t rb = (root / (2 * TBW)) * TBW + (root % TBW);
                e[k] = (m << 12) | rb;
                if (root == s) {
                    int dy, dx;
                    first_px(m, dy, dx);
                    const int y = 2 * r + dy, x = 2 * c + dx;
                    atomicOr(&RB[y][x >> 5], 1u << (x & 31));
                }
            }
            uint4 v;
            v.x = e[0] | (e[1] << 16); v.y = e[2] | (e[3] << 16);
            v.z = e[4] | (e[5] << 16); v.w = e[6] | (e[7] << 16);
            *reinterpret_cast<uint4 *>(lab + t * NBLK + r * TBW + 8 * g) = v;
        }
        __syncthreads();

        // Phase D: root bitmap and segment counts out; border components -> nodes.
        for (int i = tid; i < TH * (TW / 32); i += K1_NT) w.rbits[t * (TH * (TW / 32)) + i] = (&RB[0][0])[i];
        if (tid < TH && tid < nrp) {
            uint32_t cnt = 0;
#pragma unroll
            for (int k = 0; k < TW / 32; ++k) cnt += __popc(RB[tid][k]);
            w.segcnt[im.seg_base + int64_t(y0 + tid) * im.tiles_x + tx] = uint8_t(cnt);
        }
        uint32_t prb[(NPERIM + K1_NT - 1) / K1_NT];   // root block of each border position held
#pragma unroll
        for (int i = 0; i < (NPERIM + K1_NT - 1) / K1_NT; ++i) {
            const int p = tid + i * K1_NT;
            int r, c;
            prb[i] = kNone;
            if (p >= NPERIM || !perim_pos(p, nbr, nbc, r, c)) continue;
            const uint32_t m = M[r * TBW + c];
            if (!m) continue;
            const uint32_t root = sfind_ro(P, slot_of(r, c, m));
            const uint32_t rb = (root / (2 * TBW)) * TBW + (root % TBW);
            prb[i] = rb | (m << 16);
            atomicOr(&BF[rb >> 5], 1u << (rb & 31));
        }
        __syncthreads();
        uint32_t nb;
        const uint32_t pre = block_exscan<K1_NT>(tid < NBLK / 32 ? __popc(BF[tid]) : 0u, tmp, &nb);
        if (tid < NBLK / 32) BP[tid] = pre;
        __syncthreads();
        // Every border position writes its entry and (redundantly, with identical values) the
        // record of the node its root belongs to, which spreads the node work over the CTA.
#pragma unroll
        for (int i = 0; i < (NPERIM + K1_NT - 1) / K1_NT; ++i) {
            const int p = tid + i * K1_NT;
            if (p >= NPERIM) continue;
            uint16_t ent = 0;
            if (prb[i] != kNone) {
                const uint32_t rb = prb[i] & 0xFFFFu, m = prb[i] >> 16;
                const uint32_t j = BP[rb >> 5] + __popc(BF[rb >> 5] & ((1u << (rb & 31)) - 1u));
                ent = uint16_t((j << 4) | m);
                int dy, dx;
                first_px(M[rb], dy, dx);
                const int y = 2 * int(rb / TBW) + dy, x = 2 * int(rb % TBW) + dx;
                uint32_t rank = __popc(RB[y][x >> 5] & ((1u << (x & 31)) - 1u));
                for (int k = 0; k < (x >> 5); ++k) rank += __popc(RB[y][k]);
                const int64_t node = t * MAXB + j;
                w.nroot[node] = uint16_t(rb);
                w.nkey[node] = uint32_t(int64_t(y0 + y) * im.cols + (x0 + x));
                w.nlrank[node] = uint16_t(rank);
                w.gp[node] = uint32_t(node);
            }
            w.perim[t * NPERIM + p] = ent;
        }
        if (tid == 0) w.nb[t] = nb;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Cross-tile merge.
// ---------------------------------------------------------------------------------------------
namespace {

__device__ __forceinline__ void link_dec(const Img2D &im, Work &w, uint32_t key)
{
    const int64_t y = key / uint32_t(im.cols), x = key - y * im.cols;
    dec_u8(w.segcnt, im.seg_base + y * im.tiles_x + x / TW);
}

// Union of two nodes of one image; the root with the larger key is linked under the other.
__device__ void gunion2d(const Img2D &im, Work &w, uint32_t a, uint32_t b)
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
            link_dec(im, w, ka);
            return;
        }
    }
}

}  // namespace

constexpr int K2_NT = TBH + TBW;
constexpr int kFilterSlots2 = 2048;
constexpr int kGQ2 = 512;   // queued global unions per tile (more are done at once)

// One thread per right-border and bottom-border position.  Every connected pair goes through the
// CTA-local node filter (NodeFilter, be_common.cuh); the pairs that join two local sets are
// unioned globally from a shared queue once the tile's pairs are all seen.
__global__ void __launch_bounds__(K2_NT) k_merge_2d(ImgList2D L, Work w)
{
    __shared__ uint32_t qslot;
    __shared__ NodeFilter<kFilterSlots2> flt;
    __shared__ uint2 gq[kGQ2];
    ItemLoop loop{w.queue ? w.queue + 1 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img2D im = L.get(t);
        const int64_t lt = t - im.tile_base;
        const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
        const int nbr = (min(TH, im.rows - ty * TH) + 1) >> 1;
        const int nbc = (min(TW, im.cols - tx * TW) + 1) >> 1;
        const int p = threadIdx.x;
        const uint16_t *pe = w.perim;
        filter_reset(flt);
        __syncthreads();
        auto pair = [&](uint32_t nA, uint32_t nB) {
            if (!filter_pair(flt, nA, nB)) return;
            const uint32_t slot = atomicAdd(&flt.nq, 1u);
            if (slot < uint32_t(kGQ2)) gq[slot] = make_uint2(nA, nB);
            else gunion2d(im, w, nA, nB);
        };
        if (p < TBH) {
            // Right border: neighbours in the tile to the right, same tile row.
            const int r = p;
            const uint32_t A = (r < nbr && tx + 1 < im.tiles_x) ? pe[t * NPERIM + 2 * TBW + TBH + r] : 0u;
            if (A) {
                const uint32_t mA = A & 15u, nA = uint32_t(t * MAXB + (A >> 4));
                const int64_t t2 = t + 1;
                uint32_t last = kNone;
#pragma unroll
                for (int d = -1; d <= 1; ++d) {
                    const int rr = r + d;
                    if (rr < 0 || rr >= nbr) continue;
                    const uint32_t B = pe[t2 * NPERIM + 2 * TBW + rr];
                    if (!B) continue;
                    const uint32_t mB = B & 15u;
                    const bool c = d == 0 ? ((mA & 0xAu) && (mB & 0x5u))
                                          : d < 0 ? ((mA & 2u) && (mB & 4u)) : ((mA & 8u) && (mB & 1u));
                    const uint32_t nB = uint32_t(t2 * MAXB + (B >> 4));
                    if (c && nB != last) pair(nA, nB);
                    if (c) last = nB;
                }
            }
        } else {
            // Bottom border: neighbours in the tile row below (including the diagonal tiles).
            const int c = p - TBH;
            const uint32_t A = (c < nbc && ty + 1 < im.tiles_y) ? pe[t * NPERIM + TBW + c] : 0u;
            if (A) {
                const uint32_t mA = A & 15u, nA = uint32_t(t * MAXB + (A >> 4));
                uint32_t last = kNone;
#pragma unroll
                for (int d = -1; d <= 1; ++d) {
                    int cc = c + d;
                    int64_t t2 = t + im.tiles_x;
                    if (cc < 0) {
                        if (tx == 0) continue;
                        t2 -= 1;
                        cc = TBW - 1;
                    } else if (cc >= nbc) {
                        if (tx + 1 >= im.tiles_x) continue;
                        t2 += 1;
                        cc = 0;
                    }
                    const uint32_t B = pe[t2 * NPERIM + cc];
                    if (!B) continue;
                    const uint32_t mB = B & 15u;
                    const bool cn = d == 0 ? ((mA & 0xCu) && (mB & 0x3u))
                                           : d < 0 ? ((mA & 4u) && (mB & 2u)) : ((mA & 8u) && (mB & 1u));
                    const uint32_t nB = uint32_t(t2 * MAXB + (B >> 4));
                    if (cn && nB != last) pair(nA, nB);
                    if (cn) last = nB;
                }
            }
        }
        __syncthreads();
        const uint32_t nq = min(flt.nq, uint32_t(kGQ2));
        for (uint32_t i = threadIdx.x; i < nq; i += K2_NT) gunion2d(im, w, gq[i].x, gq[i].y);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Post-merge ranks of the surviving border roots (one CTA per tile).
// ---------------------------------------------------------------------------------------------
__device__ void post_tile_2d(const ImgList2D &L, Work &w, int64_t t)
{
    __shared__ uint32_t LB[TH][TW / 32];   // first pixels of the tile's linked nodes
    const Img2D im = L.get(t);
    const int64_t lt = t - im.tile_base;
    const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
    const int y0 = ty * TH, x0 = tx * TW;
    const uint32_t nb = w.nb[t];
    for (int i = threadIdx.x; i < TH * (TW / 32); i += blockDim.x) (&LB[0][0])[i] = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const int64_t node = t * MAXB + j;
        if (w.gp[node] == uint32_t(node)) continue;
        const uint32_t k = w.nkey[node];
        const uint32_t y = k / uint32_t(im.cols);
        const int ly = int(y) - y0, lx = int(k - y * uint32_t(im.cols)) - x0;
        atomicOr(&LB[ly][lx >> 5], 1u << (lx & 31));
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const int64_t node = t * MAXB + j;
        if (w.gp[node] != uint32_t(node)) continue;
        const uint32_t k = w.nkey[node];
        const uint32_t y = k / uint32_t(im.cols);
        const int ly = int(y) - y0, lx = int(k - y * uint32_t(im.cols)) - x0;
        uint32_t cnt = __popc(LB[ly][lx >> 5] & ((1u << (lx & 31)) - 1u));
        for (int q = 0; q < (lx >> 5); ++q) cnt += __popc(LB[ly][q]);
        w.grank[node] = w.nlrank[node] - cnt;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Label resolve and write.
// ---------------------------------------------------------------------------------------------
constexpr int K3_NT = 256;
constexpr int RBWORDS = TH * (TW / 32);   // root-bitmap words per tile
constexpr int RW = TW / 32;               // root-bitmap words per pixel row

__global__ void __launch_bounds__(K3_NT) k_tile_write_2d(ImgList2D L, Work w)
{
    __shared__ __align__(16) uint16_t Ls[NBLK];
    __shared__ uint32_t LT[NBLK];
    __shared__ uint32_t RB[RBWORDS];
    __shared__ uint32_t segb[TH];
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x, lane = tid & 31;
    const uint16_t *lab = reinterpret_cast<const uint16_t *>(w.lab);
    ItemLoop loop{w.queue ? w.queue + 4 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img2D im = L.get(t);
        const int64_t lt = t - im.tile_base;
        const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
        const int y0 = ty * TH, x0 = tx * TW;
        const int nrp = min(TH, im.rows - y0), ncp = min(TW, im.cols - x0);
        const uint32_t base0 = w.segpref[im.seg_base];

        for (int i = tid; i < NBLK / 8; i += K3_NT)
            reinterpret_cast<uint4 *>(Ls)[i] = reinterpret_cast<const uint4 *>(lab + t * NBLK)[i];
        for (int i = tid; i < RBWORDS; i += K3_NT) RB[i] = w.rbits[t * RBWORDS + i];
        if (tid < TH && tid < nrp)
            segb[tid] = w.segpref[im.seg_base + int64_t(y0 + tid) * im.tiles_x + tx] - base0;
        if (lt == 0 && tid == 0)
            w.ncomp[im.index] = int64_t(w.segpref[im.seg_base + int64_t(im.rows) * im.tiles_x] - base0);
        __syncthreads();

        // Border roots linked under another tile's root are not roots any more.
        const uint32_t nb = w.nb[t];
        for (uint32_t j = tid; j < nb; j += K3_NT) {
            const int64_t node = t * MAXB + j;
            if (w.gp[node] == uint32_t(node)) continue;
            const uint32_t rb = w.nroot[node];
            int dy, dx;
            first_px(Ls[rb] >> 12, dy, dx);
            const int y = 2 * int(rb / TBW) + dy, x = 2 * int(rb % TBW) + dx;
            atomicAnd(&RB[y * (TW / 32) + (x >> 5)], ~(1u << (x & 31)));
        }
        __syncthreads();

        // Surviving roots: rank = roots before it in its row segment.  RW consecutive lanes hold
        // the RW words of one pixel row; a shuffle scan gives each word's prefix.
        for (int i = tid; i < RBWORDS; i += K3_NT) {
            const uint32_t word = RB[i];
            uint32_t pre = __popc(word);
#pragma unroll
            for (int o = 1; o < RW; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, pre, o);
                if ((lane & (RW - 1)) >= o) pre += v;
            }
            pre -= __popc(word);
            const int y = i / RW, q = i % RW;
            const uint32_t base = 1u + segb[y] + pre;
            uint32_t bits = word;
            while (bits) {
                const int b = __ffs(bits) - 1;
                const int x = 32 * q + b;
                LT[(y >> 1) * TBW + (x >> 1)] = base + __popc(word & ((1u << b) - 1u));
                bits &= bits - 1;
            }
        }
        for (uint32_t j = tid; j < nb; j += K3_NT) {
            const int64_t node = t * MAXB + j;
            if (w.gp[node] == uint32_t(node)) continue;
            const uint32_t g = gfind_ro(w.gp, uint32_t(node));
            const uint32_t kg = w.nkey[g];
            const int64_t yg = kg / uint32_t(im.cols), xg = kg - yg * im.cols;
            const uint32_t sb = w.segpref[im.seg_base + yg * im.tiles_x + xg / TW] - base0;
            LT[w.nroot[node]] = 1u + sb + w.grank[g];
        }
        __syncthreads();

        // Output: one unit = two horizontally adjacent blocks = 4 pixels in each of 2 rows.
        const bool vec_ok = ((reinterpret_cast<uintptr_t>(im.out) | uintptr_t(im.out_pitch * 4)) & 15) == 0;
        for (int u = tid; u < NBLK / 2; u += K3_NT) {
            const int br = u / (TBW / 2), q = u % (TBW / 2);
            const int y = 2 * br;
            if (y >= nrp || 4 * q >= ncp) continue;
            const uint32_t ee = reinterpret_cast<const uint32_t *>(Ls)[u];
            const uint32_t e0 = ee & 0xFFFFu, e1 = ee >> 16;
            const uint32_t m0 = e0 >> 12, m1 = e1 >> 12;
            const int l0 = m0 ? int(LT[e0 & 0xFFFu]) : 0, l1 = m1 ? int(LT[e1 & 0xFFFu]) : 0;
            int4 a, b;
            a.x = (m0 & 1u) ? l0 : 0; a.y = (m0 & 2u) ? l0 : 0;
            a.z = (m1 & 1u) ? l1 : 0; a.w = (m1 & 2u) ? l1 : 0;
            b.x = (m0 & 4u) ? l0 : 0; b.y = (m0 & 8u) ? l0 : 0;
            b.z = (m1 & 4u) ? l1 : 0; b.w = (m1 & 8u) ? l1 : 0;
            int32_t *dst = im.out + int64_t(y0 + y) * im.out_pitch + x0 + 4 * q;
            const bool row2 = y + 1 < nrp;
            if (vec_ok && 4 * q + 4 <= ncp) {
                __stcs(reinterpret_cast<int4 *>(dst), a);
                if (row2) __stcs(reinterpret_cast<int4 *>(dst + im.out_pitch), b);
            } else {
                const int n = min(4, ncp - 4 * q);
                const int va[4] = {a.x, a.y, a.z, a.w}, vb[4] = {b.x, b.y, b.z, b.w};
                for (int k = 0; k < n; ++k) {
                    dst[k] = va[k];
                    if (row2) dst[im.out_pitch + k] = vb[k];
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Post-merge pass: border-root ranks (items < n_tiles) and scan-chunk sums (the rest).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kPostThreads) k_post_2d(ImgList2D L, Work w)
{
    __shared__ uint32_t tmp[kPostThreads / 32 + 1];
    __shared__ uint32_t qslot;
    const int64_t n = w.n_tiles + w.n_chunks;
    ItemLoop loop{w.queue ? w.queue + 2 : nullptr, n};
    for (int64_t it = loop.first(&qslot); it < n; it = loop.next(it, &qslot)) {
        if (it < w.n_tiles) post_tile_2d(L, w, it);
        else chunk_sum<kPostThreads>(w, it - w.n_tiles, tmp);
    }
}


// ---------------------------------------------------------------------------------------------
// Geometry and launch sequence of this tile shape.
// ---------------------------------------------------------------------------------------------
inline Geometry geometry()
{
    Geometry g;
    g.lab_bytes_per_tile = size_t(NBLK) * sizeof(uint16_t);
    g.rbits_bytes_per_tile = size_t(RBWORDS) * sizeof(uint32_t);
    g.nperim = NPERIM;
    g.maxb = MAXB;
    return g;
}

inline cudaError_t launch(const ImgList2D &L, const Work &w, int sms, bool persistent, cudaStream_t s,
                          cudaEvent_t *ev)
{
    auto grid = [&](int64_t items, int per_sm) -> unsigned {
        int64_t g = persistent ? std::min<int64_t>(items, int64_t(sms) * per_sm) : items;
        return unsigned(std::max<int64_t>(g, 1));
    };
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], s);
    };
    Work wk = w;
    if (!persistent) wk.queue = nullptr;
    mark(0);
    k_tile_local_2d<<<grid(w.n_tiles, 4), K1_NT, 0, s>>>(L, wk);
    mark(1);
    k_merge_2d<<<grid(w.n_tiles, 8), K2_NT, 0, s>>>(L, wk);
    mark(2);
    k_post_2d<<<grid(w.n_tiles + w.n_chunks, 12), kPostThreads, 0, s>>>(L, wk);
    mark(3);
    k_segscan<<<unsigned(std::max(w.n_chunks, 1)), kScanThreads, 0, s>>>(wk);
    mark(4);
    k_tile_write_2d<<<grid(w.n_tiles, 6), K3_NT, 0, s>>>(L, wk);
    mark(5);
    return cudaGetLastError();
}

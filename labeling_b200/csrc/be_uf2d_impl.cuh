// be_uf2d_impl.cuh -- the 2D union-find pipeline for one tile shape.  Included by be_uf2d.cu
// once per supported shape, inside a namespace that defines `TBW` and `TBH` (tile width and
// height in 2x2 blocks, TBW * TBH <= 4096, TBW a power of two in [64, 256]).
namespace {

constexpr int TW = 2 * TBW, TH = 2 * TBH;          // tile in pixels
constexpr int NBLK = TBW * TBH;                    // blocks per tile (4096)
constexpr int NPERIM = 2 * (TBW + TBH);            // border positions per tile
constexpr int MAXB = NPERIM;                       // nodes per tile
constexpr int WPR = TBW / 32;                      // 32-block words per block row
constexpr int K1_NT = TBH * WPR;                   // one thread per (block row, word) = NBLK / 32
constexpr int MQCAP = 608;                         // union-queue capacity (more take further rounds)
constexpr uint32_t kPass = 0xFFFFu;                // "no run start" in the carry scan

static_assert(NBLK <= 4096, "tile-local block index must fit 12 bits");
static_assert(MAXB < 4096, "node index must fit 12 bits");
static_assert(K1_NT == NBLK / 32 && (WPR & (WPR - 1)) == 0 && WPR <= 32, "thread layout");

// Union-find slot order of a block: r*2*TBW + t*TBW + c with t = 0 when the block has a pixel in
// its top row.  The order is the raster order of the blocks' first pixels, so the smallest slot
// of a component is the block holding its first pixel.  Mask bits: 0 = top-left, 1 = top-right,
// 2 = bottom-left, 3 = bottom-right pixel.
__device__ __forceinline__ uint32_t key_block(uint32_t key)
{
    return (key / (2 * TBW)) * TBW + (key % TBW);
}

// Pixel offset (row, column) of a block's first foreground pixel, inside the block.
__device__ __forceinline__ void first_px(uint32_t m, int &dy, int &dx)
{
    if (m & 3u) { dy = 0; dx = (m & 1u) ? 0 : 1; }
    else { dy = 1; dx = (m & 4u) ? 0 : 1; }
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

// Byte-wise x > thr for four pixels: bit 7 of each byte.  K = 0x7F - (thr & 0x7F) in every byte;
// `hi` = thr >= 128.  (x & 0x7F) + K carries into bit 7 exactly when the low seven bits exceed
// thr's; the high bit decides the rest.
__device__ __forceinline__ uint32_t gt_bytes(uint32_t x, uint32_t K, bool hi)
{
    const uint32_t s = (x & 0x7F7F7F7Fu) + K;
    return (hi ? (x & s) : (x | s)) & 0x80808080u;
}

// Bits 7, 15, 23, 31 -> bits 0..3 (the four partial products land on distinct bits, no carries).
__device__ __forceinline__ uint32_t gather4(uint32_t g) { return (g * 0x00204081u) >> 28; }

// 16 pixels of one row -> foreground bits of their even (left) and odd (right) pixels: 8 blocks.
__device__ __forceinline__ void split16(uint4 v, uint32_t K, bool hi, uint32_t &ev, uint32_t &od)
{
    ev = gather4(gt_bytes(__byte_perm(v.x, v.y, 0x6420), K, hi)) |
         (gather4(gt_bytes(__byte_perm(v.z, v.w, 0x6420), K, hi)) << 4);
    od = gather4(gt_bytes(__byte_perm(v.x, v.y, 0x7531), K, hi)) |
         (gather4(gt_bytes(__byte_perm(v.z, v.w, 0x7531), K, hi)) << 4);
}

// Bits 0..3 of x -> bit 0 of bytes 0..3.
__device__ __forceinline__ uint32_t spread4(uint32_t x) { return ((x & 0xFu) * 0x00204081u) & 0x01010101u; }

// Highest set bit of x (x != 0).
__device__ __forceinline__ uint32_t hibit(uint32_t x) { return 31u - __clz(x); }

// Shared-memory position of block x's union-find entry: the low five bits are XOR-ed with the
// block's 32-block word, so that the 32 lanes of a warp -- 32 different words walking the same
// bit position -- reach 32 different banks.  Entries still name blocks by their plain index.
__device__ __forceinline__ uint32_t sw(uint32_t x) { return x ^ ((x >> 5) & 31u); }

// Union-find over run starts with the slot order carried in the parent entry: P[x] holds
// (slot << 12) | parent, and a root holds its own (slot << 12) | x.  Entries only ever decrease,
// so the union (atomicMin of the smaller encoding into the other root, Playne-Hawick style)
// leaves the run with the smallest slot -- the component's first pixel -- as the root.
__device__ __forceinline__ uint32_t efind(uint32_t *P, uint32_t x)
{
    uint32_t v = P[sw(x)];
    while ((v & 0xFFFu) != x) {
        const uint32_t y = v & 0xFFFu;
        const uint32_t vg = P[sw(y)];
        if ((vg & 0xFFFu) != y) P[sw(x)] = vg;   // path halving
        x = y;
        v = vg;
    }
    return x;
}

__device__ __forceinline__ uint32_t efind_ro(const uint32_t *P, uint32_t x)
{
    uint32_t v = P[sw(x)];
    while ((v & 0xFFFu) != x) {
        x = v & 0xFFFu;
        v = P[sw(x)];
    }
    return x;
}

// As efind, also returning the root's own entry as read (the union compares the two).
__device__ __forceinline__ uint32_t efind_e(uint32_t *P, uint32_t x, uint32_t &ev)
{
    uint32_t v = P[sw(x)];
    while ((v & 0xFFFu) != x) {
        const uint32_t y = v & 0xFFFu;
        const uint32_t vg = P[sw(y)];
        if ((vg & 0xFFFu) != y) P[sw(x)] = vg;
        x = y;
        v = vg;
    }
    ev = v;
    return x;
}

__device__ __forceinline__ void eunion(uint32_t *P, uint32_t a, uint32_t b)
{
    for (;;) {
        uint32_t ea, eb;
        a = efind_e(P, a, ea);
        b = efind_e(P, b, eb);
        if (a == b) return;
        if (ea < eb) {
            const uint32_t old = atomicMin(&P[sw(b)], ea);
            if ((old & 0xFFFu) == b) return;
            b = old & 0xFFFu;
        } else {
            const uint32_t old = atomicMin(&P[sw(a)], eb);
            if ((old & 0xFFFu) == a) return;
            a = old & 0xFFFu;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Tile-local labeling.  One thread per 32 blocks of a block row (a "word"): the four pixel
// classes of the blocks (top-left, top-right, bottom-left, bottom-right) are 32-bit words, so
// horizontal runs of joined blocks, their starts and the links to the row above are bitwise
// operations; only runs enter the union-find, and only links between runs that no earlier link
// already joins are merged.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(K1_NT, 8) k_tile_local_2d(ImgList2D L, Work w)
{
    grid_dep_release();   // the merge launch may take free SMs during this grid's last wave
    if (blockIdx.x == 0 && threadIdx.x == 0) {   // a new epoch for the segment scan of this run
        w.epoch[0] += 1u;
        w.epoch[1] = 0u;
    }
    __shared__ uint32_t P[NBLK];            // run starts: (slot << 12) | parent
    __shared__ __align__(16) uint8_t M[NBLK];
    __shared__ uint32_t WBL[NBLK / 32], WBR[NBLK / 32], WHC[NBLK / 32], WS[NBLK / 32], WCS[NBLK / 32];
    __shared__ uint32_t RB[TH][TW / 32];
    __shared__ uint32_t BF[NBLK / 32];
    __shared__ uint32_t MQ[MQCAP];          // union queue: (block_a << 16) | block_b
    static_assert(MQCAP >= NBLK / 32, "the node numbering reuses the queue's memory");
    uint32_t *const BP = MQ;                // node numbering per 32 blocks (after the unions)
    __shared__ uint32_t mqn;
    __shared__ uint32_t tmp[K1_NT / 32 + 1];
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x;
    const int r = tid / WPR, q = tid % WPR;
    uint16_t *lab = reinterpret_cast<uint16_t *>(w.lab);
    ItemLoop loop{w.queue ? w.queue + 0 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img2D im = L.get(t);
        const int64_t lt = t - im.tile_base;
        const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
        const int y0 = ty * TH, x0 = tx * TW;
        const int nrp = min(TH, im.rows - y0), ncp = min(TW, im.cols - x0);
        const int nbr = (nrp + 1) >> 1, nbc = (ncp + 1) >> 1;
        const uint32_t K = (0x7Fu - (uint32_t(im.thr) & 0x7Fu)) * 0x01010101u;
        const bool hi = im.thr >= 128;

        for (int i = tid; i < TH * (TW / 32); i += K1_NT) (&RB[0][0])[i] = 0;
        BF[tid] = 0;
        if (tid == 0) mqn = 0;

        // Phase A: pixel words, runs, run starts and their slots.
        uint32_t TLw = 0, TRw = 0, BLw = 0, BRw = 0;
        if (r < nbr && 64 * q < ncp) {
            const uint8_t *row0 = im.in + int64_t(y0 + 2 * r) * im.in_pitch + x0 + 64 * q;
            const bool row1 = 2 * r + 1 < nrp;
            const bool vec = (64 * q + 64 <= ncp) &&
                             ((reinterpret_cast<uintptr_t>(row0) | uintptr_t(im.in_pitch)) & 15) == 0;
            if (vec) {
                const uint4 *p0 = reinterpret_cast<const uint4 *>(row0);
                uint4 v[4], u[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) v[i] = __ldg(p0 + i);
                if (row1) {
                    const uint4 *p1 = reinterpret_cast<const uint4 *>(row0 + im.in_pitch);
#pragma unroll
                    for (int i = 0; i < 4; ++i) u[i] = __ldg(p1 + i);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    uint32_t ev, od;
                    split16(v[i], K, hi, ev, od);
                    TLw |= ev << (8 * i);
                    TRw |= od << (8 * i);
                    if (row1) {
                        split16(u[i], K, hi, ev, od);
                        BLw |= ev << (8 * i);
                        BRw |= od << (8 * i);
                    }
                }
            } else {
                const int n = min(64, ncp - 64 * q);
                for (int x = 0; x < n; ++x) {
                    const uint32_t bt = uint32_t(row0[x] > im.thr) << (x >> 1);
                    const uint32_t bb = row1 ? uint32_t(row0[im.in_pitch + x] > im.thr) << (x >> 1) : 0u;
                    if (x & 1) { TRw |= bt; BRw |= bb; }
                    else { TLw |= bt; BLw |= bb; }
                }
            }
        }
        const uint32_t Lw = TLw | BLw, Rw = TRw | BRw, Tw = TLw | TRw, Fw = Tw | BLw | BRw;
        // hc bit k: block k is joined to block k + 1 (a right pixel of k touches a left pixel of
        // k + 1 -- every such pair is 8-adjacent); bit 31 looks at the next word.
        const uint32_t Lnext = __shfl_down_sync(0xFFFFFFFFu, Lw, 1, WPR);
        const uint32_t hc = (Rw & (Lw >> 1)) | ((q + 1 < WPR) ? (Rw & (Lnext << 31)) : 0u);
        const uint32_t hcprev = __shfl_up_sync(0xFFFFFFFFu, hc, 1, WPR);
        const uint32_t cin = q > 0 ? (hcprev >> 31) : 0u;   // block 0 continues a run from the left
        const uint32_t hl = (hc << 1) | cin;                  // bit k: block k joined to block k - 1
        const uint32_t S = Fw & ~hl;                          // run starts
        // Column of the start of the run entering from the left: the last start among the words
        // before this one (an inclusive "last start" scan over the row's words).
        uint32_t v = S ? uint32_t(32 * q) + hibit(S) : kPass;
#pragma unroll
        for (int o = 1; o < WPR; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, v, o, WPR);
            if (q >= o && v == kPass) v = u;
        }
        const uint32_t vprev = __shfl_up_sync(0xFFFFFFFFu, v, 1, WPR);
        const uint32_t CSc = cin ? vprev : kPass;
        const uint32_t rbase = uint32_t(r) * TBW, sbase = uint32_t(r) * (2 * TBW);

        // Block masks as bytes (for the first-pixel lookups and the border entries).
        uint32_t mw[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int k = 4 * i;
            mw[i] = spread4(TLw >> k) | (spread4(TRw >> k) << 1) | (spread4(BLw >> k) << 2) |
                    (spread4(BRw >> k) << 3);
        }
        {
            uint4 *mdst = reinterpret_cast<uint4 *>(&M[rbase + 32 * q]);
            mdst[0] = make_uint4(mw[0], mw[1], mw[2], mw[3]);
            mdst[1] = make_uint4(mw[4], mw[5], mw[6], mw[7]);
        }
        WBL[tid] = BLw;
        WBR[tid] = BRw;
        WHC[tid] = hc;
        WS[tid] = S;
        WCS[tid] = CSc;
        // Slot keys across words: a run that goes on into later words of its row takes its slot
        // from the first top pixel there when its own part has none.  Each word reports the first
        // top pixel of the run carried into it (0xFF: none) and whether that run also goes on past
        // the word (0x100); the word holding the run's start reads them with shuffles inside the
        // row's lanes, so every slot is complete when it is first written.
        const uint32_t cbrk = ~hc;
        const uint32_t ctm = cin ? (Tw & ((2u << (cbrk ? uint32_t(__ffs(cbrk) - 1) : 31u)) - 1u)) : 0u;
        const uint32_t mine = (ctm ? uint32_t(32 * q + __ffs(ctm) - 1) : 0xFFu) | ((cin && !cbrk) ? 0x100u : 0u);
        uint32_t tail = 0xFFu;   // first top pixel of this word's last run in the words after it
        {
            bool open = (hc >> 31) & 1u;   // the word's last run goes on into the next word
#pragma unroll
            for (int d = 1; d < WPR; ++d) {
                const uint32_t pj = __shfl_down_sync(0xFFFFFFFFu, mine, d, WPR);
                if (open && q + d < WPR) {
                    if ((pj & 0xFFu) != 0xFFu) {
                        tail = pj & 0xFFu;
                        open = false;
                    } else if (!(pj & 0x100u)) {
                        open = false;
                    }
                }
            }
        }
        __syncthreads();   // words of every row written

        // Phase B: links to the block row above.  For block b of this row: N (straight up, a top
        // pixel over a bottom pixel), NW (top-left pixel to the bottom-right pixel of b - 1 above)
        // and NE (top-right to the bottom-left pixel of b + 1 above).  A link is dropped when an
        // earlier link (further left, or N before NW / NE at the same block) joins the same two
        // runs; every chain of such reasons ends at a link that is kept.
        uint32_t Nm = 0, NWm = 0, NEm = 0;
        if (r > 0 && r < nbr) {
            const int u = tid - WPR;   // same word, row above
            const uint32_t uBL = WBL[u], uBR = WBR[u];
            const uint32_t uBRp = q > 0 ? WBR[u - 1] >> 31 : 0u;
            const uint32_t uBLn = q + 1 < WPR ? WBL[u + 1] & 1u : 0u;
            const uint32_t N = Tw & (uBL | uBR);
            const uint32_t NW = TLw & ((uBR << 1) | uBRp);
            const uint32_t NE = TRw & ((uBL >> 1) | (uBLn << 31));
            Nm = N; NWm = NW; NEm = NE;
        }
        {
            // bit 31 of the previous word's raw N / NE, for the rules at block 0
            const uint32_t Np = __shfl_up_sync(0xFFFFFFFFu, Nm, 1, WPR);
            const uint32_t NEp = __shfl_up_sync(0xFFFFFFFFu, NEm, 1, WPR);
            if (r > 0 && r < nbr) {
                const int u = tid - WPR;
                const uint32_t uhc = WHC[u];
                const uint32_t uhl = (uhc << 1) | (q > 0 ? WHC[u - 1] >> 31 : 0u);
                const uint32_t N = Nm, NE = NEm;
                const uint32_t Nsh = (N << 1) | (q > 0 ? Np >> 31 : 0u);
                const uint32_t NEsh = (NE << 1) | (q > 0 ? NEp >> 31 : 0u);
                Nm = N & ~(hl & ((Nsh & uhl) | NEsh));
                NWm &= ~((N & uhl) | (hl & Nsh));
                NEm = NE & ~((N & uhc) | (hl & NEsh & uhc));
            }
        }
        // The run start of a block: a start in the block's word at or before it, else the start
        // carried in from the left.
        auto start_of = [&](uint32_t blk) -> uint32_t {
            const uint32_t m = WS[blk >> 5] & ((2u << (blk & 31u)) - 1u);
            const uint32_t st = m ? (blk & ~31u) + hibit(m) : (blk & ~uint32_t(TBW - 1)) + WCS[blk >> 5];
            // A start of this tile by construction; the mask only keeps a broken invariant
            // from leaving the array.
            (void)GUARD(w, st < uint32_t(NBLK), 112, (uint64_t(blk) << 32) | st);
            return st & (NBLK - 1);
        };
        const uint32_t ubase = rbase - TBW + 32 * q, abase = rbase + 32 * q;

        // Every run that starts in this word gets its entry.  A run with a kept link in this word
        // takes the first one as its parent: the parent is in the row above, whose slots are all
        // smaller than this row's, so a plain store links it (no atomic, no cycle possible).  Its
        // entry holds key 0 -- the smallest value, so no atomicMin of a union ever changes it and
        // unions walk on to the parent; only a root's key is ever compared.  Any other run is a
        // root for now: (slot << 12) | itself, the slot being its first block with a top pixel
        // (this word, else the words after it), else its start.  These forest links leave the
        // queue; the union-find below walks the forest like any other path (path halving), and
        // the flatten pass compresses it.  (Pointer jumping over the forest first was measured
        // slower.)
        {
            uint32_t ss = S;
            while (ss) {
                const uint32_t s0 = __ffs(ss) - 1;
                ss &= ss - 1;
                const uint32_t from = ~0u << s0;
                const uint32_t brk = ~hc & from;
                const uint32_t e = brk ? uint32_t(__ffs(brk) - 1) : 31u;
                const uint32_t span = from & (0xFFFFFFFFu >> (31u - e));
                const uint32_t lk = (Nm | NWm | NEm) & span;
                const uint32_t x = abase + s0;
                if (lk) {
                    const uint32_t b = __ffs(lk) - 1, bit = 1u << b;
                    uint32_t tgt;
                    if (Nm & bit) {
                        tgt = ubase + b;
                        Nm &= ~bit;
                    } else if (NWm & bit) {
                        tgt = ubase + b - 1;
                        NWm &= ~bit;
                    } else {
                        tgt = ubase + b + 1;
                        NEm &= ~bit;
                    }
                    P[sw(x)] = start_of(tgt);   // key 0
                } else {
                    const uint32_t tm = Tw & span;
                    uint32_t key = sbase + TBW + 32 * q + s0;
                    if (tm) key = sbase + 32 * q + (__ffs(tm) - 1);
                    else if (brk == 0 && tail != 0xFFu) key = sbase + tail;
                    P[sw(x)] = (key << 12) | x;
                }
            }
        }
        // The remaining links are unions.  The queue holds the two blocks of each link; their run
        // starts are looked up by the merging lanes, which share that work evenly.  Links past the
        // queue's capacity go in in later rounds.
        const uint32_t n = __popc(Nm) + __popc(NWm) + __popc(NEm);
        const uint32_t pos0 = warp_reserve(&mqn, n);
        auto each_link = [&](auto &&f) {
            uint32_t pos = pos0;
            uint32_t todo = Nm | NWm | NEm;
            while (todo) {
                const uint32_t b = __ffs(todo) - 1;
                todo &= todo - 1;
                const uint32_t bit = 1u << b;
                const uint32_t a = abase + b;
                if (Nm & bit) f(pos++, a, ubase + b);
                if (NWm & bit) f(pos++, a, ubase + b - 1);   // b = 0: the last block of the word before
                if (NEm & bit) f(pos++, a, ubase + b + 1);   // b = 31: the first block of the word after
            }
        };
        if (pos0 < uint32_t(MQCAP))
            each_link([&](uint32_t pos, uint32_t a, uint32_t b) {
                if (pos < uint32_t(MQCAP)) MQ[pos] = (a << 16) | b;
            });
        __syncthreads();
        // Rounds of the queue: the links with positions [base, base + MQCAP) go in, and each thread
        // takes a contiguous run of them: neighbouring links, mostly of the same rows, are merged
        // one after another by one thread instead of racing on the same roots.
        {
            const uint32_t total = mqn;
            for (uint32_t base = 0; base < total; base += MQCAP) {
                if (base) {
                    if (pos0 + n > base && pos0 < base + MQCAP)
                        each_link([&](uint32_t pos, uint32_t a, uint32_t b) {
                            if (pos >= base && pos < base + MQCAP) MQ[pos - base] = (a << 16) | b;
                        });
                    __syncthreads();
                }
                const uint32_t nq = min(total - base, uint32_t(MQCAP));
                const uint32_t per = (nq + K1_NT - 1) / K1_NT, lo = min(nq, uint32_t(tid) * per), hi = min(nq, lo + per);
                for (uint32_t i = lo; i < hi; ++i) eunion(P, start_of(MQ[i] >> 16), start_of(MQ[i] & 0xFFFFu));
                __syncthreads();
            }
        }

        // Phase C: every run start of this word is pointed straight at its root (a read-only walk,
        // then the root's entry stored in the start's own entry; every entry is a run start, so each
        // is compressed by its own thread, and no link happens any more -- storing the root along
        // the walked path as well was measured slower: a second dependent walk); roots mark their
        // first pixel.  Then the block entries: (mask << 12) | root block, two blocks per 32-bit word.
        {
            uint32_t ss = S;
            while (ss) {
                const uint32_t x = abase + (__ffs(ss) - 1);
                ss &= ss - 1;
                uint32_t root = x, ev = P[sw(x)];
                for (int it = 0; (ev & 0xFFFu) != root && it < NBLK; ++it) {   // acyclic: the cap never binds
                    root = ev & 0xFFFu;
                    ev = P[sw(root)];
                }
                if (root != x) P[sw(x)] = ev;
                if (root == x) {
                    const uint32_t key = ev >> 12;
                    const uint32_t rb = key_block(key);
                    int dy, dx;
                    first_px(M[rb], dy, dx);
                    const int y = 2 * int(key / (2 * TBW)) + dy, xx = 2 * int(key % TBW) + dx;
                    atomicOr(&RB[y][xx >> 5], 1u << (xx & 31));
                }
            }
        }
        {
            uint32_t cur = 0;
            if (cin) {   // the run carried in from the left starts in an earlier word of this row
                uint32_t root = rbase + (CSc & (TBW - 1)), ev = P[sw(root)];
                for (int it = 0; (ev & 0xFFFu) != root && it < NBLK; ++it) {
                    root = ev & 0xFFFu;
                    ev = P[sw(root)];
                }
                cur = key_block(ev >> 12);
            }
            uint32_t ew[16];
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                if ((S >> k) & 1u) cur = key_block(P[sw(abase + k)] >> 12);
                const uint32_t m = (mw[k >> 2] >> (8 * (k & 3))) & 15u;
                const uint32_t e = m ? (m << 12) | cur : 0u;
                if (k & 1) ew[k >> 1] |= e << 16;
                else ew[k >> 1] = e;
            }
            uint4 *dst = reinterpret_cast<uint4 *>(lab + t * NBLK + abase);
#pragma unroll
            for (int i = 0; i < 4; ++i) dst[i] = make_uint4(ew[4 * i], ew[4 * i + 1], ew[4 * i + 2], ew[4 * i + 3]);
        }
        __syncthreads();   // root bitmap complete; every run start points at its root

        // Phase D: root bitmap and segment counts out; border components -> nodes.
        for (int i = tid; i < TH * (TW / 32); i += K1_NT) w.rbits[t * (TH * (TW / 32)) + i] = (&RB[0][0])[i];
        if (tid < TH && tid < nrp) {
            uint32_t cnt = 0;
#pragma unroll
            for (int k = 0; k < TW / 32; ++k) cnt += __popc(RB[tid][k]);
            w.segcnt[im.seg_base + int64_t(y0 + tid) * im.tiles_x + tx] = uint8_t(cnt);
        }
        // Root block of each border position held (plus its mask, and whether this position
        // claimed the node: the one position that sets the root's bit writes the node's record).
        constexpr uint32_t kOwner = 1u << 20;
        uint32_t prb[(NPERIM + K1_NT - 1) / K1_NT];
#pragma unroll
        for (int i = 0; i < (NPERIM + K1_NT - 1) / K1_NT; ++i) {
            const int p = tid + i * K1_NT;
            int br, bc;
            prb[i] = kNone;
            if (p >= NPERIM || !perim_pos(p, nbr, nbc, br, bc)) continue;
            const uint32_t m = M[br * TBW + bc];
            if (!m) continue;
            const int wi = br * WPR + (bc >> 5);
            const uint32_t sm = WS[wi] & ((2u << (bc & 31)) - 1u);
            const uint32_t sc = sm ? uint32_t(bc & ~31) + hibit(sm) : WCS[wi];
            (void)GUARD(w, sc < uint32_t(TBW), 113, sc);
            const uint32_t rb = key_block(P[sw(uint32_t(br) * TBW + (sc & (TBW - 1)))] >> 12);
            const uint32_t bit = 1u << (rb & 31);
            const uint32_t old = atomicOr(&BF[rb >> 5], bit);
            prb[i] = rb | (m << 16) | ((old & bit) ? 0u : kOwner);
        }
        __syncthreads();
        uint32_t nb;
        const uint32_t pre = block_exscan<K1_NT>(__popc(BF[tid]), tmp, &nb);
        BP[tid] = pre;
        __syncthreads();
            // Every border position writes its entry; the position that claimed its node writes the
        // node's record.
#pragma unroll
        for (int i = 0; i < (NPERIM + K1_NT - 1) / K1_NT; ++i) {
            const int p = tid + i * K1_NT;
            if (p >= NPERIM) continue;
            uint16_t ent = 0;
            if (prb[i] != kNone) {
                const uint32_t rb = prb[i] & 0xFFFFu, m = (prb[i] >> 16) & 15u;
                const uint32_t j = BP[rb >> 5] + __popc(BF[rb >> 5] & ((1u << (rb & 31)) - 1u));
                ent = uint16_t((j << 4) | m);
            }
            if (prb[i] != kNone && (prb[i] & kOwner)) {
                const uint32_t rb = prb[i] & 0xFFFFu;
                const uint32_t j = BP[rb >> 5] + __popc(BF[rb >> 5] & ((1u << (rb & 31)) - 1u));
                int dy, dx;
                first_px(M[rb], dy, dx);
                const int y = 2 * int(rb / TBW) + dy, x = 2 * int(rb % TBW) + dx;
                const int64_t node = t * MAXB + j;
                const uint32_t key = uint32_t(int64_t(y0 + y) * im.cols + (x0 + x));
                w.nroot[node] = uint16_t(rb);
                w.gp[node] = gentry(key, uint32_t(node));
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

// A root linked under another leaves its segment's root count and the root bitmap of its tile
// (so that after the merge the bitmaps hold exactly the components' first pixels).
__device__ __forceinline__ void link_dec(const Img2D &im, Work &w, uint32_t key)
{
    const int64_t y = key / uint32_t(im.cols), x = key - y * im.cols;
    const int64_t ty = y / TH, tx = x / TW;
    dec_u8(w.segcnt, im.seg_base + y * im.tiles_x + tx);
    const int ly = int(y - ty * TH), lx = int(x - tx * TW);
    atomicAnd(w.rbits + (im.tile_base + ty * im.tiles_x + tx) * (TH * (TW / 32)) + ly * (TW / 32) + (lx >> 5),
              ~(1u << (lx & 31)));
}

// Union of two nodes of one image; the root with the larger key is linked under the other, and
// the linked root leaves its segment's root count and its tile's root bitmap.
__device__ void gunion2d(const Img2D &im, Work &w, uint32_t a, uint32_t b)
{
    gunion_keyed(w.gp, a, b, [&](uint32_t key) { link_dec(im, w, key); });
}

}  // namespace

constexpr int K2_NP = TBH + TBW;               // border positions a merge CTA looks at
constexpr int K2_NT = 64;                      // threads of a merge CTA (small: many tiles per SM)
constexpr int K2_PER_SM = 28;                  // resident merge CTAs per SM
constexpr int kGQ2 = 256;                      // queued global unions per tile (more are done at once)
constexpr int SR = MAXB;                       // local index of the staged right column
constexpr int SD = MAXB + TBH;                 // local index of the staged bottom row (column -1 first)
constexpr int NLOC2 = MAXB + TBH + TBW + 2;    // local union-find size

// Positions p < TBH are the right border's rows, the others the bottom border's columns
// (p - TBH).  The border entries across the right border (the next tile's left column) and the
// bottom border (the top row of the tile below, widened by one block into the two diagonal tiles)
// are staged in shared memory with the global node id they belong to.  A CTA-local union-find over
// this tile's nodes and the staged positions (neighbouring staged positions of one node merged
// first) filters the pairs: only a pair that joins two local sets goes on to the global
// union-find, from a shared queue once all of the tile's pairs are seen.  The merge is bound by
// the latency of those global unions (dependent L2 round trips), so a CTA is two warps that loop
// over the positions: many tiles are in flight on each SM at once.
__global__ void __launch_bounds__(K2_NT, K2_PER_SM) k_merge_2d(ImgList2D L, Work w)
{
    grid_dep_wait();
    grid_dep_release();
    __shared__ uint32_t qslot;
    __shared__ uint32_t lp[NLOC2];
    __shared__ uint32_t sid[TBH + TBW + 2];   // staged global node ids (kNone = none)
    __shared__ uint8_t smk[TBH + TBW + 2];    // staged masks
    __shared__ uint16_t own[K2_NP];           // this tile's own border entries
    __shared__ uint8_t cm[K2_NP];             // connected staged neighbours of each position
    __shared__ uint2 gq[kGQ2];
    __shared__ uint32_t nq;
    ItemLoop loop{w.queue ? w.queue + 1 : nullptr, w.n_tiles};
    for (int64_t t = loop.first(&qslot); t < w.n_tiles; t = loop.next(t, &qslot)) {
        const Img2D im = L.get(t);
        const int64_t lt = t - im.tile_base;
        const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
        const int nbr = (min(TH, im.rows - ty * TH) + 1) >> 1;
        const int nbc = (min(TW, im.cols - tx * TW) + 1) >> 1;
        const uint16_t *pe = w.perim;
        for (int i = threadIdx.x; i < NLOC2; i += K2_NT) lp[i] = uint32_t(i);
        if (threadIdx.x == 0) nq = 0;
        // Stage: position p < TBH stages right-column row p; the others bottom-row column p - TBH,
        // and the first two of those also columns -1 and TBW.  Each position's own entry is loaded
        // with the staging loads.
        auto stage = [&](int k, int64_t t2, int pos) {
            const uint32_t B = pe[t2 * NPERIM + pos];
            sid[k] = B ? uint32_t(t2 * MAXB + (B >> 4)) : kNone;
            smk[k] = uint8_t(B & 15u);
        };
        for (int p = threadIdx.x; p < K2_NP; p += K2_NT) {
            uint16_t A = 0;
            if (p < TBH) {
                if (p < nbr && tx + 1 < im.tiles_x) {
                    A = pe[t * NPERIM + 2 * TBW + TBH + p];
                    stage(p, t + 1, 2 * TBW + p);
                } else {
                    sid[p] = kNone;
                    smk[p] = 0;
                }
            } else {
                const int c = p - TBH;
                const int k = TBH + 1 + c;
                if (c < nbc && ty + 1 < im.tiles_y) {
                    A = pe[t * NPERIM + TBW + c];
                    stage(k, t + im.tiles_x, c);
                } else {
                    sid[k] = kNone;
                    smk[k] = 0;
                }
                if (c == 0) {
                    if (tx > 0 && ty + 1 < im.tiles_y) stage(TBH, t + im.tiles_x - 1, TBW - 1);
                    else { sid[TBH] = kNone; smk[TBH] = 0; }
                }
                if (c == 1) {
                    // column TBW: block 0 of the tile below-right (a tile with a right neighbour is
                    // full-width; a narrower tile's column nbc is staged empty by its own position)
                    if (nbc == TBW && tx + 1 < im.tiles_x && ty + 1 < im.tiles_y)
                        stage(TBH + TBW + 1, t + im.tiles_x + 1, 0);
                    else { sid[TBH + TBW + 1] = kNone; smk[TBH + TBW + 1] = 0; }
                }
            }
            own[p] = A;
        }
        __syncthreads();
        // Neighbouring staged positions of one node are one element: every position of a run of
        // equal node ids along the staged column (warp 0) or row (warp 1) points at the run's first
        // position, found by ballots 32 positions at a time (no merging, no chains).
        {
            const int lane = threadIdx.x & 31;
            const int lo = threadIdx.x < 32 ? 0 : TBH, n = threadIdx.x < 32 ? TBH : TBW + 2;
            uint32_t carry = 0;
            for (int c0 = 0; c0 < n; c0 += 32) {
                const int k = c0 + lane;
                const bool valid = k < n;
                const bool start = valid && (k == 0 || sid[lo + k] != sid[lo + k - 1]);
                const uint32_t below = __ballot_sync(0xFFFFFFFFu, start) & (0xFFFFFFFFu >> (31 - lane));
                const uint32_t st = below ? uint32_t(c0) + hibit(below) : carry;
                if (valid) lp[MAXB + lo + k] = uint32_t(MAXB + lo) + st;
                carry = __shfl_sync(0xFFFFFFFFu, st, 31);
            }
        }
        // Connected neighbours of every position: bit d + 1 for the staged neighbour at offset d.
        for (int p = threadIdx.x; p < K2_NP; p += K2_NT) {
            const uint32_t A = own[p];
            uint32_t cb = 0;
            if (A) {
                const uint32_t mA = A & 15u;
                if (p < TBH) {
                    // Right border: neighbours in the tile to the right, same tile row.
#pragma unroll
                    for (int d = -1; d <= 1; ++d) {
                        const int rr = p + d;
                        if (rr < 0 || rr >= nbr || sid[rr] == kNone) continue;
                        const uint32_t mB = smk[rr];
                        if (d == 0 ? ((mA & 0xAu) && (mB & 0x5u)) : d < 0 ? ((mA & 2u) && (mB & 4u)) : ((mA & 8u) && (mB & 1u)))
                            cb |= 1u << (d + 1);
                    }
                } else {
                    // Bottom border: neighbours in the tile row below (including the diagonal tiles).
                    const int c = p - TBH;
#pragma unroll
                    for (int d = -1; d <= 1; ++d) {
                        const int k = c + d + 1;   // staged bottom index
                        if (sid[TBH + k] == kNone) continue;
                        const uint32_t mB = smk[TBH + k];
                        if (d == 0 ? ((mA & 0xCu) && (mB & 0x3u)) : d < 0 ? ((mA & 4u) && (mB & 2u)) : ((mA & 8u) && (mB & 1u)))
                            cb |= 1u << (d + 1);
                    }
                }
            }
            cm[p] = uint8_t(cb);
        }
        __syncthreads();
        // Pairs.  Staged index of a position's neighbour at offset d: p + d on the right border,
        // TBH + c + d + 1 on the bottom border.  A pair is skipped when the position before (same
        // border, same own node) touches the same staged run: that position's pair stands for it.
        // A pair that passes goes through the CTA-local union-find, and only one that joins two
        // local sets goes on to the global union-find.
        auto pair = [&](uint32_t ja, uint32_t nA, uint32_t le, uint32_t nB) {
            if (!smerge_joined(lp, ja, le)) return;
            const uint32_t slot = atomicAdd(&nq, 1u);
            if (slot < uint32_t(kGQ2)) gq[slot] = make_uint2(nA, nB);
            else gunion2d(im, w, nA, nB);
        };
        for (int p = threadIdx.x; p < K2_NP; p += K2_NT) {
            const uint32_t A = own[p];
            uint32_t cb = cm[p];
            if (!A || !cb) continue;
            const uint32_t ja = A >> 4, nA = uint32_t(t * MAXB + ja);
            const int i0 = p < TBH ? p : p + 1;   // staged index of the neighbour at offset d: i0 + d
            // the position before on the same border, when it belongs to the same own node
            const bool prev = p != 0 && p != TBH && own[p - 1] && (own[p - 1] >> 4) == ja;
            const uint32_t cbp = prev ? cm[p - 1] : 0u;
            uint32_t lastB = kNone;   // a node already paired with this one needs no second pair
            while (cb) {
                const int d = __ffs(cb) - 2;
                cb &= cb - 1;
                const int i = i0 + d;
                const uint32_t nB = sid[i], rs = lp[MAXB + i];
                if (nB == lastB) continue;
                bool seen = false;
#pragma unroll
                for (int dp = -1; dp <= 1; ++dp)
                    if ((cbp >> (dp + 1)) & 1u) seen |= lp[MAXB + i0 - 1 + dp] == rs;
                if (seen) continue;
                pair(ja, nA, rs, nB);
                lastB = nB;
            }
        }
        __syncthreads();
        const uint32_t nqt = min(nq, uint32_t(kGQ2));
        for (uint32_t i = threadIdx.x; i < nqt; i += K2_NT) gunion2d(im, w, gq[i].x, gq[i].y);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Segment scan and node flatten, one launch: items below n_chunks scan a chunk of segment counts
// (single pass, look-back); the others point every linked node of one tile straight at its global
// root (flatten_tile_nodes: all unions are done; the nodes of all tiles jump at once), so that the
// label writes find each root in one step however long the merge's chains grew.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kScanThreads) k_scan_flatten_2d(Work w)
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
        flatten_tile_nodes(w, it - w.n_chunks, MAXB);
    }
}

// ---------------------------------------------------------------------------------------------
// Label resolve and write.
// ---------------------------------------------------------------------------------------------
constexpr int K3_NT = 256;
constexpr int RBWORDS = TH * (TW / 32);   // root-bitmap words per tile
constexpr int RW = TW / 32;               // root-bitmap words per pixel row

__global__ void __launch_bounds__(K3_NT, 8) k_tile_write_2d(ImgList2D L, Work w)
{
    __shared__ __align__(16) uint16_t Ls[NBLK];
    __shared__ uint32_t LT[NBLK];
    __shared__ uint32_t RB[RBWORDS];
    __shared__ uint32_t segb[TH];
    __shared__ uint32_t qslot;

    const int tid = threadIdx.x, lane = tid & 31;
    const uint16_t *lab = reinterpret_cast<const uint16_t *>(w.lab);
    // Block entries and the root bitmap (first pixels of the components that stayed roots through
    // the merge) were final before this grid's predecessor (segment scan and node flatten) started:
    // that grid waits for the merge to complete before it lets this one launch.  So they are read
    // before the wait (through L2), and only the segment prefixes, which the scan writes, after it.
    // With a fixed tile order (no work queue) the CTA loads the next tile's entries, bitmap and
    // node count into registers while it writes the current tile's labels.
    static_assert(NBLK / 8 == 2 * K3_NT && RBWORDS == 2 * K3_NT, "two prefetched words per thread");
    uint4 nL[2];
    uint32_t nR[2], nNb = 0;
    auto fetch = [&](int64_t t) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            nL[i] = __ldcg(reinterpret_cast<const uint4 *>(lab + t * NBLK) + tid + i * K3_NT);
            nR[i] = __ldcg(w.rbits + t * RBWORDS + tid + i * K3_NT);
        }
        nNb = __ldcg(w.nb + t);
    };
    const bool fixed_order = w.queue == nullptr;
    ItemLoop loop{w.queue ? w.queue + 4 : nullptr, w.n_tiles};
    int64_t t = loop.first(&qslot);
    if (t < w.n_tiles) fetch(t);
    for (bool first = true; t < w.n_tiles; t = loop.next(t, &qslot), first = false) {
        if (!fixed_order && !first) fetch(t);   // a work queue gives the next tile only now
        const Img2D im = L.get(t);
        const int64_t lt = t - im.tile_base;
        const int ty = int(lt / im.tiles_x), tx = int(lt - int64_t(ty) * im.tiles_x);
        const int y0 = ty * TH, x0 = tx * TW;
        const int nrp = min(TH, im.rows - y0), ncp = min(TW, im.cols - x0);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            reinterpret_cast<uint4 *>(Ls)[tid + i * K3_NT] = nL[i];
            RB[tid + i * K3_NT] = nR[i];
        }
        const uint32_t nb = nNb;
        if (fixed_order && t + gridDim.x < w.n_tiles) fetch(t + gridDim.x);
        grid_dep_wait();   // segment prefixes from here on (returns at once after the first tile)
        const uint32_t base0 = w.segpref[im.seg_base];
        if (tid < TH && tid < nrp)
            segb[tid] = w.segpref[im.seg_base + int64_t(y0 + tid) * im.tiles_x + tx] - base0;
        if (lt == 0 && tid == 0)
            w.ncomp[im.index] = int64_t(w.segpref[im.seg_base + int64_t(im.rows) * im.tiles_x] - base0);
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
        // Border components linked under another tile's component: the label of that root, its
        // segment's prefix plus its rank among the first pixels left in its row of its tile.
        for (uint32_t j = tid; j < nb; j += K3_NT) {
            const int64_t node = t * MAXB + j;
            if (uint32_t(__ldcg(w.gp + node)) == uint32_t(node)) continue;
            const uint32_t g = gfind_halve(w.gp, uint32_t(node));
            const uint32_t kg = uint32_t(__ldcg(w.gp + g) >> 32);
            const int64_t yg = kg / uint32_t(im.cols), xg = kg - yg * im.cols;
            const int64_t tyg = yg / TH, txg = xg / TW;
            const int ly = int(yg - tyg * TH), lx = int(xg - txg * TW);
            const uint32_t *rw = w.rbits + (im.tile_base + tyg * im.tiles_x + txg) * RBWORDS + ly * RW;
            uint32_t rank = __popc(__ldcg(rw + (lx >> 5)) & ((1u << (lx & 31)) - 1u));
            for (int k = 0; k < (lx >> 5); ++k) rank += __popc(__ldcg(rw + k));
            const uint32_t sb = w.segpref[im.seg_base + yg * im.tiles_x + txg] - base0;
            LT[__ldcg(w.nroot + node)] = 1u + sb + rank;
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
    // The launches after the first overlap their start with the tail of the one before (they
    // wait for it on the device); not when events are recorded between them.
    const bool ov = !persistent && !ev;
    cudaError_t e = cudaSuccess;
    auto keep = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    mark(0);
    k_tile_local_2d<<<grid(w.n_tiles, 8), K1_NT, 0, s>>>(L, wk);
    keep(cudaGetLastError());
    mark(1);
    keep(launch_k(k_merge_2d, grid(w.n_tiles, K2_PER_SM), K2_NT, s, ov, L, wk));
    mark(2);
    keep(launch_k(k_scan_flatten_2d, grid(int64_t(w.n_chunks) + w.n_tiles, 8), kScanThreads, s, ov, wk));
    mark(3);
    // The label writes run a fixed tile order over 8 CTAs per SM (they prefetch their next tile).
    keep(launch_k(k_tile_write_2d, unsigned(std::max<int64_t>(1, std::min<int64_t>(w.n_tiles, int64_t(sms) * 8))),
                  K3_NT, s, ov, L, wk));
    mark(4);
    return e;
}

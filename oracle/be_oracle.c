/*
 * be_oracle.c -- CPU oracle for Block-Equivalence (BE) connected-component labeling.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path (labeling_b200/, include/) links,
 * loads or calls this file.  It is used by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py, always as the checker, never as the thing measured.
 *
 * Contents (plain C99, single-threaded):
 *   orc_be2d_raw  restatement of the reference 2D GPU BE path: host padding of
 *                 IOCLLabeling::Label (Labeling2015/src/LabelingTools.cpp:98-132) and the
 *                 LBEQ2_Init / LBEQ2_Scan / LBEQ2_Analyze / LBEQ2_SetFinalLabels kernels
 *                 (Labeling2015/src/LabelingAlgs.cl:176-319) driven by the host loop of
 *                 TOCLLabelEquivalenceX2 (Labeling2015/src/LabelingAlgs.cpp:989-1084).
 *                 Output: the reference's own label values (1 + smallest block index of the
 *                 component in the padded block grid), cropped to rows x cols.
 *   orc_be3d_raw  the same for 3D: IOCLLabeling3D::Label + CopyAlignImg
 *                 (LabelingTools.cpp:160-221) and BLEQ3D_* (LabelingAlgs.cl:740-979) driven by
 *                 TOCLBlockEquivalence3D (LabelingAlgs.cpp:1443-1536).  Output cropped back to
 *                 the unpadded d0 x d1 x d2 volume (the reference returns the padded volume).
 *   orc_lbeq2d_raw / orc_lbeq3d_raw
 *                 restatement of the pixel-level label-equivalence path selected by -a lbeq -g:
 *                 DistrInitKernel/DistrScanKernel/DistrAnalizeKernel (LabelingAlgs.cl:31-130,
 *                 host LabelingAlgs.cpp:867-942) and LBEQ3D_* (LabelingAlgs.cl:635-734, host
 *                 LabelingAlgs.cpp:1324-1396).
 *   orc_canon     canonical relabeling: components numbered 1..K by first foreground pixel in
 *                 raster order, background 0.  Returns K.
 *   orc_ccl2d / orc_ccl3d
 *                 independent union-find labeling (8- / 26-connectivity, or 4 / 6 when asked)
 *                 that emits canonical labels directly.  It is a second, fast oracle for sizes
 *                 where the BE emulation (serial root chase) is too slow.
 *
 * Foreground is `pixel > thr`.  The reference binarizes with cv::threshold(img, img, 8, 255,
 * THRESH_BINARY) (LabelingTools.cpp:46: THRESH_OTSU == 8 is passed as the threshold value and
 * CV_8UC1 == 0 as the type), i.e. thr = 8; its kernels then test `pixel != 0` (thr = 0).
 *
 * Uninitialised device memory in the reference: LBEQ2_Init / BLEQ3D_Init write sLabels only for
 * non-empty blocks (LabelingAlgs.cl:201-202, 827-828) into buffers made by clCreateBuffer without a
 * host pointer (LabelingAlgs.cpp:996, 1451), and the 2D padding rows/columns come from an
 * uninitialised cv::Mat (LabelingTools.cpp:103).  The algorithm needs zeros in both places; this
 * restatement zero-fills them.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_EINVAL -1
#define ORC_ENOMEM -2

/* ------------------------------------------------------------------------------------------ */
/* 2D Block Equivalence                                                                        */
/* ------------------------------------------------------------------------------------------ */

/* Neighbour-block offsets in the reference's connectivity-bit order: bit k of sConn refers to
 * block (x + DX2[k], y + DY2[k]) (LabelingAlgs.cl:163-167 layout, 243-250 use). */
static const int DX2[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
static const int DY2[8] = {-1, -1, -1, 0, 0, 1, 1, 1};

/* 1 when the padded image has a foreground pixel at (x, y); 0 outside the buffer. */
static inline int px2(const uint8_t *p, int64_t W, int64_t H, int64_t x, int64_t y)
{
    if (x < 0 || y < 0 || x >= W || y >= H) return 0;
    return p[y * W + x] != 0;
}

/* LBEQ2_Init (LabelingAlgs.cl:176-227): a block's bit k is set when a foreground pixel of the
 * block is 8-adjacent to a foreground pixel of neighbour block k.  The reference encodes this
 * with the 4x4 "testPattern" (union of the 3x3 neighbourhoods of the block's foreground pixels)
 * and tests the neighbour pixels that fall inside it; RemoveBorderBlocks (:151-159) drops the
 * pattern column/row that would fall outside the image.  The explicit adjacency test below is
 * the same predicate with bounds checks instead of border masks. */
static uint8_t be2d_conn(const uint8_t *p, int64_t W, int64_t H, int64_t bx, int64_t by)
{
    uint8_t conn = 0;
    for (int k = 0; k < 8; ++k) {
        int hit = 0;
        for (int i = 0; i < 4 && !hit; ++i) {
            int64_t ax = 2 * bx + (i & 1), ay = 2 * by + (i >> 1);
            if (!px2(p, W, H, ax, ay)) continue;
            for (int j = 0; j < 4 && !hit; ++j) {
                int64_t qx = 2 * (bx + DX2[k]) + (j & 1), qy = 2 * (by + DY2[k]) + (j >> 1);
                int64_t ddx = qx - ax, ddy = qy - ay;
                if (ddx < -1 || ddx > 1 || ddy < -1 || ddy > 1) continue;
                if (px2(p, W, H, qx, qy)) hit = 1;
            }
        }
        if (hit) conn |= (uint8_t)(1u << k);
    }
    return conn;
}

int orc_be2d_raw(const uint8_t *img, int64_t rows, int64_t cols, int64_t pitch, int thr,
                 uint32_t *out)
{
    if (rows <= 0 || cols <= 0 || pitch < cols || !img || !out) return ORC_EINVAL;
    /* IOCLLabeling::Label padding (LabelingTools.cpp:103-104). */
    const int64_t W = (cols >> 5 << 5) + 32, H = (rows >> 5 << 5) + 32;
    const int64_t SW = (W + 1) / 2, SH = (H + 1) / 2; /* InitSPixels (LabelingAlgs.cpp:993-994) */
    uint8_t *p = (uint8_t *)calloc((size_t)(W * H), 1);
    uint32_t *sl = (uint32_t *)calloc((size_t)(SW * SH), sizeof(uint32_t));
    uint8_t *sc = (uint8_t *)calloc((size_t)(SW * SH), 1);
    if (!p || !sl || !sc) { free(p); free(sl); free(sc); return ORC_ENOMEM; }
    for (int64_t y = 0; y < rows; ++y)
        for (int64_t x = 0; x < cols; ++x)
            p[y * W + x] = img[y * pitch + x] > thr ? 255 : 0;

    /* LBEQ2_Init over the {SW, SH} NDRange. */
    for (int64_t by = 0; by < SH; ++by)
        for (int64_t bx = 0; bx < SW; ++bx) {
            int64_t s = bx + by * SW;
            int nonempty = px2(p, W, H, 2 * bx, 2 * by) | px2(p, W, H, 2 * bx + 1, 2 * by) |
                           px2(p, W, H, 2 * bx, 2 * by + 1) | px2(p, W, H, 2 * bx + 1, 2 * by + 1);
            if (nonempty) {
                sl[s] = (uint32_t)(s + 1);
                sc[s] = be2d_conn(p, W, H, bx, by);
            }
        }

    /* LabelSPixels host loop (LabelingAlgs.cpp:1028-1038): Scan until no change, Analyze. */
    for (;;) {
        int no_changes = 1;
        /* LBEQ2_Scan (LabelingAlgs.cl:257-280) with MinSPixLabel (:239-253). */
        for (int64_t by = 0; by < SH; ++by)
            for (int64_t bx = 0; bx < SW; ++bx) {
                int64_t s = bx + by * SW;
                uint32_t label = sl[s];
                if (!label) continue;
                uint32_t m = UINT32_MAX;
                for (int k = 0; k < 8; ++k)
                    if (sc[s] & (1u << k)) {
                        uint32_t v = sl[(bx + DX2[k]) + (by + DY2[k]) * SW];
                        if (v < m) m = v;
                    }
                if (m < label) {
                    if (m < sl[label - 1]) sl[label - 1] = m;
                    no_changes = 0;
                }
            }
        if (no_changes) break;
        /* LBEQ2_Analyze (LabelingAlgs.cl:284-300): chase to the self-referencing root. */
        for (int64_t s = 0; s < SW * SH; ++s) {
            uint32_t label = sl[s];
            if (!label) continue;
            uint32_t cur = sl[label - 1];
            while (cur != label) {
                label = sl[cur - 1];
                cur = sl[label - 1];
            }
            sl[s] = label;
        }
    }

    /* LBEQ2_SetFinalLabels (LabelingAlgs.cl:304-319), then the crop of LabelingTools.cpp:129. */
    for (int64_t y = 0; y < rows; ++y)
        for (int64_t x = 0; x < cols; ++x)
            out[y * cols + x] = p[y * W + x] ? sl[(x >> 1) + (y >> 1) * SW] : 0;
    free(p); free(sl); free(sc);
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------------ */
/* 3D Block Equivalence                                                                        */
/* ------------------------------------------------------------------------------------------ */

/* 1 when the padded volume has a foreground voxel at (x, y, z) (x = dim 0, z = dim 2 fastest). */
static inline int vx3(const uint8_t *v, int64_t X, int64_t Y, int64_t Z, int64_t x, int64_t y,
                      int64_t z)
{
    if (x < 0 || y < 0 || z < 0 || x >= X || y >= Y || z >= Z) return 0;
    return v[(x * Y + y) * Z + z] != 0;
}

/* BLEQ3D_Init (LabelingAlgs.cl:805-860): bit (dx+1) + 3(dy+1) + 9(dz+1) of sConn is set when a
 * foreground voxel of the block is 26-adjacent to a foreground voxel of the neighbour block at
 * (dx, dy, dz).  The reference unrolls the face/edge/corner cases as TEST_CONN4/2/1 over a 4x4x4
 * test pattern (:750-787, 830-856); this is the same predicate written as a loop. */
static uint32_t be3d_conn(const uint8_t *v, int64_t X, int64_t Y, int64_t Z, int64_t bx,
                          int64_t by, int64_t bz)
{
    uint32_t conn = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                if (!dx && !dy && !dz) continue;
                int hit = 0;
                for (int i = 0; i < 8 && !hit; ++i) {
                    int64_t ax = 2 * bx + (i >> 2), ay = 2 * by + ((i >> 1) & 1),
                            az = 2 * bz + (i & 1);
                    if (!vx3(v, X, Y, Z, ax, ay, az)) continue;
                    for (int j = 0; j < 8 && !hit; ++j) {
                        int64_t qx = 2 * (bx + dx) + (j >> 2), qy = 2 * (by + dy) + ((j >> 1) & 1),
                                qz = 2 * (bz + dz) + (j & 1);
                        int64_t ex = qx - ax, ey = qy - ay, ez = qz - az;
                        if (ex < -1 || ex > 1 || ey < -1 || ey > 1 || ez < -1 || ez > 1) continue;
                        if (vx3(v, X, Y, Z, qx, qy, qz)) hit = 1;
                    }
                }
                if (hit) conn |= 1u << ((dx + 1) + 3 * (dy + 1) + 9 * (dz + 1));
            }
    return conn;
}

int orc_be3d_raw(const uint8_t *vol, int64_t d0, int64_t d1, int64_t d2, int thr, uint32_t *out)
{
    if (d0 <= 0 || d1 <= 0 || d2 <= 0 || !vol || !out) return ORC_EINVAL;
    /* CopyAlignImg (LabelingTools.cpp:160-176): each dim to ((n + 4) >> 5 << 5) + 32, data at +2. */
    const int64_t X = ((d0 + 4) >> 5 << 5) + 32, Y = ((d1 + 4) >> 5 << 5) + 32,
                  Z = ((d2 + 4) >> 5 << 5) + 32;
    const int64_t SX = X >> 1, SY = Y >> 1, SZ = Z >> 1; /* InitSPixels (LabelingAlgs.cpp:1447-1449) */
    const int64_t NS = SX * SY * SZ;
    uint8_t *v = (uint8_t *)calloc((size_t)(X * Y * Z), 1);
    uint32_t *sl = (uint32_t *)calloc((size_t)NS, sizeof(uint32_t));
    uint32_t *sc = (uint32_t *)calloc((size_t)NS, sizeof(uint32_t));
    if (!v || !sl || !sc) { free(v); free(sl); free(sc); return ORC_ENOMEM; }
    for (int64_t x = 0; x < d0; ++x)
        for (int64_t y = 0; y < d1; ++y)
            for (int64_t z = 0; z < d2; ++z)
                v[((x + 2) * Y + (y + 2)) * Z + (z + 2)] = vol[(x * d1 + y) * d2 + z] > thr ? 255 : 0;

    for (int64_t bx = 0; bx < SX; ++bx)
        for (int64_t by = 0; by < SY; ++by)
            for (int64_t bz = 0; bz < SZ; ++bz) {
                int64_t s = (bx * SY + by) * SZ + bz;
                int nonempty = 0;
                for (int i = 0; i < 8; ++i)
                    nonempty |= vx3(v, X, Y, Z, 2 * bx + (i >> 2), 2 * by + ((i >> 1) & 1),
                                    2 * bz + (i & 1));
                if (nonempty) {
                    sl[s] = (uint32_t)(s + 1);
                    sc[s] = be3d_conn(v, X, Y, Z, bx, by, bz);
                }
            }

    for (;;) {
        int no_changes = 1;
        /* BLEQ3D_Scan (LabelingAlgs.cl:904-932) with MinSPixLabel3D (:872-900). */
        for (int64_t bx = 0; bx < SX; ++bx)
            for (int64_t by = 0; by < SY; ++by)
                for (int64_t bz = 0; bz < SZ; ++bz) {
                    int64_t s = (bx * SY + by) * SZ + bz;
                    uint32_t label = sl[s];
                    if (!label) continue;
                    uint32_t m = UINT32_MAX;
                    for (int k = 0; k < 27; ++k) {
                        if (k == 13 || !(sc[s] & (1u << k))) continue;
                        int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
                        uint32_t val = sl[((bx + dx) * SY + (by + dy)) * SZ + (bz + dz)];
                        if (val < m) m = val;
                    }
                    if (m < label) {
                        if (m < sl[label - 1]) sl[label - 1] = m;
                        no_changes = 0;
                    }
                }
        if (no_changes) break;
        /* BLEQ3D_Analyze (LabelingAlgs.cl:936-952). */
        for (int64_t s = 0; s < NS; ++s) {
            uint32_t label = sl[s];
            if (!label) continue;
            uint32_t cur = sl[label - 1];
            while (cur != label) {
                label = sl[cur - 1];
                cur = sl[label - 1];
            }
            sl[s] = label;
        }
    }

    /* BLEQ3D_SetFinalLabels (LabelingAlgs.cl:956-979), cropped back to the input volume. */
    for (int64_t x = 0; x < d0; ++x)
        for (int64_t y = 0; y < d1; ++y)
            for (int64_t z = 0; z < d2; ++z) {
                int64_t px = x + 2, py = y + 2, pz = z + 2;
                uint32_t lab = 0;
                if (v[(px * Y + py) * Z + pz])
                    lab = sl[((px >> 1) * SY + (py >> 1)) * SZ + (pz >> 1)];
                out[(x * d1 + y) * d2 + z] = lab;
            }
    free(v); free(sl); free(sc);
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------------ */
/* Pixel-level label equivalence (-a lbeq -g)                                                  */
/* ------------------------------------------------------------------------------------------ */

/* MinLabel (LabelingAlgs.cl:54-62) returns the smaller non-zero label and UINT_MAX when both are
 * zero; the nested MinLabel chains of MinNWSELabel / Min3DLabel therefore yield the smallest
 * non-zero neighbour label, or UINT_MAX when there is none.  Folding with `acc` starting at
 * UINT_MAX gives the same value. */
static inline uint32_t lbeq_min(uint32_t acc, uint32_t v)
{
    return (v && v < acc) ? v : acc;
}

/* DistrInit/Scan/Analize (LabelingAlgs.cl:31-130) over a rows x cols image (the host pads it
 * like IOCLLabeling::Label, LabelingTools.cpp:103).  Labels are 0-based pixel positions and
 * GetLabel (:48-50) treats position 0 as background, so a foreground pixel at (0, 0) keeps label 0
 * and is reported as background -- the reference behaviour, reproduced here on purpose.
 * conn8 != 0 selects the 8-neighbour scan (coh == COH_8, :68); the reference's default
 * (COH_DEFAULT) takes the 4-neighbour branch. */
int orc_lbeq2d_raw(const uint8_t *img, int64_t rows, int64_t cols, int64_t pitch, int thr,
                   int conn8, uint32_t *out)
{
    if (rows <= 0 || cols <= 0 || pitch < cols || !img || !out) return ORC_EINVAL;
    const int64_t W = (cols >> 5 << 5) + 32, H = (rows >> 5 << 5) + 32, N = W * H;
    uint32_t *lb = (uint32_t *)calloc((size_t)N, sizeof(uint32_t));
    if (!lb) return ORC_ENOMEM;
    for (int64_t y = 0; y < rows; ++y)
        for (int64_t x = 0; x < cols; ++x)
            if (img[y * pitch + x] > thr) lb[y * W + x] = (uint32_t)(y * W + x);
    static const int64_t OFF8[8][2] = {{-1, 0}, {0, -1}, {0, 1}, {-1, -1},
                                       {1, 1},  {-1, 1}, {1, -1}, {1, 0}};
    static const int64_t OFF4[4][2] = {{-1, 0}, {0, -1}, {0, 1}, {1, 0}};
    for (;;) {
        int no_changes = 1;
        for (int64_t pos = 0; pos < N; ++pos) {
            uint32_t label = lb[pos];
            if (!label) continue;
            /* MinNWSELabel (:66-82): GetLabel (:48-50) reads flat positions and returns 0 for
             * position 0 and positions >= W*H (rows wrap, as in the reference). */
            uint32_t m = UINT32_MAX;
            const int nn = conn8 ? 8 : 4;
            for (int k = 0; k < nn; ++k) {
                const int64_t *o = conn8 ? OFF8[k] : OFF4[k];
                int64_t q = pos + o[0] + o[1] * W;
                uint32_t val = (q > 0 && q < N) ? lb[q] : 0;
                m = lbeq_min(m, val);
            }
            if (m < label) {
                if (m < lb[label]) lb[label] = m;
                no_changes = 0;
            }
        }
        if (no_changes) break;
        for (int64_t pos = 0; pos < N; ++pos) { /* DistrAnalizeKernel (:114-130) */
            uint32_t label = lb[pos];
            if (!label) continue;
            uint32_t cur = lb[label];
            while (cur != label) {
                label = lb[cur];
                cur = lb[label];
            }
            lb[pos] = label;
        }
    }
    for (int64_t y = 0; y < rows; ++y)
        for (int64_t x = 0; x < cols; ++x) out[y * cols + x] = lb[y * W + x];
    free(lb);
    return ORC_OK;
}

/* LBEQ3D_InitKernel/ScanKernel/AnalyzeKernel (LabelingAlgs.cl:635-734) on the CopyAlignImg
 * padded volume, 1-based labels, 26 neighbours via Min3DLabel (:655-683). */
int orc_lbeq3d_raw(const uint8_t *vol, int64_t d0, int64_t d1, int64_t d2, int thr, uint32_t *out)
{
    if (d0 <= 0 || d1 <= 0 || d2 <= 0 || !vol || !out) return ORC_EINVAL;
    const int64_t X = ((d0 + 4) >> 5 << 5) + 32, Y = ((d1 + 4) >> 5 << 5) + 32,
                  Z = ((d2 + 4) >> 5 << 5) + 32, N = X * Y * Z;
    uint32_t *lb = (uint32_t *)calloc((size_t)N, sizeof(uint32_t));
    if (!lb) return ORC_ENOMEM;
    for (int64_t x = 0; x < d0; ++x)
        for (int64_t y = 0; y < d1; ++y)
            for (int64_t z = 0; z < d2; ++z)
                if (vol[(x * d1 + y) * d2 + z] > thr) {
                    int64_t pos = ((x + 2) * Y + (y + 2)) * Z + (z + 2);
                    lb[pos] = (uint32_t)(pos + 1);
                }
    for (;;) {
        int no_changes = 1;
        for (int64_t x = 0; x < X; ++x)
            for (int64_t y = 0; y < Y; ++y)
                for (int64_t z = 0; z < Z; ++z) {
                    int64_t pos = (x * Y + y) * Z + z;
                    uint32_t label = lb[pos];
                    if (!label) continue;
                    uint32_t mm = UINT32_MAX;
                    for (int dx = -1; dx <= 1; ++dx)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dz = -1; dz <= 1; ++dz) {
                                if (!dx && !dy && !dz) continue;
                                int64_t qx = x + dx, qy = y + dy, qz = z + dz;
                                uint32_t val = 0; /* GetLabel3D (:646-651) */
                                if (qx >= 0 && qy >= 0 && qz >= 0 && qx < X && qy < Y && qz < Z)
                                    val = lb[(qx * Y + qy) * Z + qz];
                                mm = lbeq_min(mm, val);
                            }
                    if (mm < label) {
                        if (mm < lb[label - 1]) lb[label - 1] = mm;
                        no_changes = 0;
                    }
                }
        if (no_changes) break;
        for (int64_t pos = 0; pos < N; ++pos) {
            uint32_t label = lb[pos];
            if (!label) continue;
            uint32_t cur = lb[label - 1];
            while (cur != label) {
                label = lb[cur - 1];
                cur = lb[label - 1];
            }
            lb[pos] = label;
        }
    }
    for (int64_t x = 0; x < d0; ++x)
        for (int64_t y = 0; y < d1; ++y)
            for (int64_t z = 0; z < d2; ++z)
                out[(x * d1 + y) * d2 + z] = lb[((x + 2) * Y + (y + 2)) * Z + (z + 2)];
    free(lb);
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------------ */
/* Canonical relabeling                                                                        */
/* ------------------------------------------------------------------------------------------ */

/* Components numbered 1..K in order of their first foreground element in flat (raster) order;
 * 0 stays background.  Returns K, or a negative error. */
int64_t orc_canon(const uint32_t *lab, int64_t n, int32_t *out)
{
    uint32_t mx = 0;
    for (int64_t i = 0; i < n; ++i)
        if (lab[i] > mx) mx = lab[i];
    int32_t *map = (int32_t *)calloc((size_t)mx + 1, sizeof(int32_t));
    if (!map) return ORC_ENOMEM;
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t l = lab[i];
        if (!l) { out[i] = 0; continue; }
        if (!map[l]) map[l] = (int32_t)(++k);
        out[i] = map[l];
    }
    free(map);
    return k;
}

/* ------------------------------------------------------------------------------------------ */
/* Independent union-find labeling (canonical output)                                          */
/* ------------------------------------------------------------------------------------------ */

static inline int64_t uf_find(int64_t *par, int64_t a)
{
    while (par[a] != a) {
        par[a] = par[par[a]];
        a = par[a];
    }
    return a;
}

static inline void uf_union(int64_t *par, int64_t a, int64_t b)
{
    a = uf_find(par, a);
    b = uf_find(par, b);
    if (a == b) return;
    if (a < b) par[b] = a;
    else par[a] = b;
}

/* Unions keep the smallest raster index as the root, so each component's root is its first
 * foreground pixel and a raster sweep numbers components canonically. */
static int64_t uf_emit(int64_t *par, const uint8_t *fg, int64_t n, int32_t *out)
{
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (!fg[i]) { out[i] = 0; continue; }
        int64_t r = uf_find(par, i);
        if (r == i) out[i] = (int32_t)(++k);
        else out[i] = out[r];
    }
    return k;
}

int64_t orc_ccl2d(const uint8_t *img, int64_t rows, int64_t cols, int64_t pitch, int thr,
                  int conn8, int32_t *out)
{
    if (rows < 0 || cols < 0 || (rows && pitch < cols)) return ORC_EINVAL;
    const int64_t n = rows * cols;
    if (n == 0) return 0;
    int64_t *par = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    uint8_t *fg = (uint8_t *)malloc((size_t)n);
    if (!par || !fg) { free(par); free(fg); return ORC_ENOMEM; }
    for (int64_t y = 0; y < rows; ++y)
        for (int64_t x = 0; x < cols; ++x) {
            fg[y * cols + x] = img[y * pitch + x] > thr;
            par[y * cols + x] = y * cols + x;
        }
    for (int64_t y = 0; y < rows; ++y)
        for (int64_t x = 0; x < cols; ++x) {
            int64_t i = y * cols + x;
            if (!fg[i]) continue;
            if (x > 0 && fg[i - 1]) uf_union(par, i, i - 1);
            if (y > 0) {
                if (fg[i - cols]) uf_union(par, i, i - cols);
                if (conn8 && x > 0 && fg[i - cols - 1]) uf_union(par, i, i - cols - 1);
                if (conn8 && x + 1 < cols && fg[i - cols + 1]) uf_union(par, i, i - cols + 1);
            }
        }
    int64_t k = uf_emit(par, fg, n, out);
    free(par); free(fg);
    return k;
}

/* conn26 != 0: 26-connectivity; otherwise 6-connectivity (faces only). */
int64_t orc_ccl3d(const uint8_t *vol, int64_t d0, int64_t d1, int64_t d2, int thr, int conn26,
                  int32_t *out)
{
    if (d0 < 0 || d1 < 0 || d2 < 0) return ORC_EINVAL;
    const int64_t n = d0 * d1 * d2;
    if (n == 0) return 0;
    int64_t *par = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    uint8_t *fg = (uint8_t *)malloc((size_t)n);
    if (!par || !fg) { free(par); free(fg); return ORC_ENOMEM; }
    for (int64_t i = 0; i < n; ++i) {
        fg[i] = vol[i] > thr;
        par[i] = i;
    }
    for (int64_t x = 0; x < d0; ++x)
        for (int64_t y = 0; y < d1; ++y)
            for (int64_t z = 0; z < d2; ++z) {
                int64_t i = (x * d1 + y) * d2 + z;
                if (!fg[i]) continue;
                /* the 13 neighbours that precede (x, y, z) in raster order */
                for (int dx = -1; dx <= 0; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = -1; dz <= 1; ++dz) {
                            if (dx == 0 && (dy > 0 || (dy == 0 && dz >= 0))) continue;
                            if (!conn26 && (dx != 0) + (dy != 0) + (dz != 0) != 1) continue;
                            int64_t qx = x + dx, qy = y + dy, qz = z + dz;
                            if (qx < 0 || qy < 0 || qz < 0 || qy >= d1 || qz >= d2) continue;
                            int64_t q = (qx * d1 + qy) * d2 + qz;
                            if (fg[q]) uf_union(par, i, q);
                        }
            }
    int64_t k = uf_emit(par, fg, n, out);
    free(par); free(fg);
    return k;
}

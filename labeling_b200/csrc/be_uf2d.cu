// be_uf2d.cu -- 2D Block-Equivalence labeling, union-find form (8-connectivity, 2x2 blocks).
// The pipeline itself is in be_uf2d_impl.cuh, instantiated here for three tile shapes
// (32 x 128, 64 x 64 and 16 x 256 blocks) that the autotuner chooses between.
//
// Replaces the reference's LBEQ2_Init / LBEQ2_Scan / LBEQ2_Analyze / LBEQ2_SetFinalLabels
// (LabelingAlgs.cl:176-319) and their host loop (LabelingAlgs.cpp:989-1084) with four launches:
//
//   k_tile_local_2d   one CTA per 64x256-pixel tile: 16-byte coalesced loads, 2x2 block masks,
//                     runs of blocks and their links by bit operations; each run's first link
//                     becomes its parent by a plain store (a forest), the other links are
//                     atomicMin unions in shared memory (smaller key wins), then every run start
//                     walks to its root;
//                     write one uint16 per block = (mask << 12) | tile-local root block; count
//                     roots per segment; mark each component's first pixel in the tile's root
//                     bitmap; export border components as nodes.
//   k_merge_2d        unions nodes across tile borders (global union-find after Rem's
//                     algorithm, smaller key wins); every root that gets linked leaves its segment
//                     count and its root bitmap.
//   k_scan_flatten_2d single-pass exclusive scan of the segment counts (be_scan.cuh) and, in
//                     the same launch, every linked node pointed at its global root (pointer
//                     jumping).
//   k_tile_write_2d   one CTA per tile: resolves each block's canonical label and writes the int32
//                     labels with 16-byte stores.
//
// Canonical numbering.  A block's key is the raster index of its first foreground pixel.  Blocks
// are merged so that every component is rooted at its smallest key, i.e. at its first pixel in
// raster order; its label is 1 + the number of component roots that precede that pixel.  The root
// counts per segment (image row x tile column) and their exclusive prefix give that number.
//
// Shared-memory union-find slots.  Within a tile the union-find runs over "slots" whose order is
// the key order: slot = r * 2*TBW + t * TBW + c for the block in block-row r, block-column c,
// where t = 0 when the block has a foreground pixel in its top pixel row and 1 otherwise.  Its
// first pixel is in pixel row 2r + t, so slot order equals raster order of first pixels, and the
// atomicMin union keeps the first pixel's block as the root.
#include "be_common.cuh"
#include "be_kernels.h"
#include "be_scan.cuh"

#include "be_api_internal.h"

#include <algorithm>

namespace be {

namespace s32x128 {
constexpr int TBW = 128, TBH = 32;
#include "be_uf2d_impl.cuh"
}  // namespace s32x128

namespace s64x64 {
constexpr int TBW = 64, TBH = 64;
#include "be_uf2d_impl.cuh"
}  // namespace s64x64

namespace s16x256 {
constexpr int TBW = 256, TBH = 16;
#include "be_uf2d_impl.cuh"
}  // namespace s16x256

const Shape2D kShapes2D[kNumShapes2D] = {{128, 32}, {64, 64}, {256, 16}};

Geometry uf2d_geometry(int shape)
{
    switch (shape) {
    case 1: return s64x64::geometry();
    case 2: return s16x256::geometry();
    default: return s32x128::geometry();
    }
}

cudaError_t uf2d_launch(int shape, const ImgList2D &L, const Work &w, int sms, bool persistent,
                        cudaStream_t s, cudaEvent_t *ev)
{
    switch (shape) {
    case 1: return s64x64::launch(L, w, sms, persistent, s, ev);
    case 2: return s16x256::launch(L, w, sms, persistent, s, ev);
    default: return s32x128::launch(L, w, sms, persistent, s, ev);
    }
}

}  // namespace be

// be_kernels.h -- kernel entry points and tile geometry shared by the host code (be_api.cu)
// and the kernel files.
#pragma once
#include "be_common.cuh"

// Default 2D tile (shape 0): 128 x 32 blocks = 256 x 64 pixels.  be_uf2d.cu also instantiates
// 64 x 64 and 256 x 16 blocks (shapes 1 and 2).
#define T2_TBW 128
#define T2_TBH 32
#define T2_NPERIM (2 * (T2_TBW + T2_TBH))
#define T2_MAXB T2_NPERIM

// 3D tile: 8 x 16 x 32 blocks = 16 x 32 x 64 voxels (d0, d1, d2).
#define T3_TB0 8
#define T3_TB1 16
#define T3_TB2 32
#define T3_NBLK (T3_TB0 * T3_TB1 * T3_TB2)
#define T3_NPERIM (2 * (T3_TB0 * T3_TB1 + T3_TB0 * T3_TB2 + T3_TB1 * T3_TB2))
#define T3_MAXB T3_NPERIM

namespace be {

__global__ void k_tile_local_3d(ImgList3D L, Work w);
__global__ void k_merge_3d(ImgList3D L, Work w);
__global__ void k_scan_link_3d(ImgList3D L, Work w);
__global__ void k_tile_write_3d(ImgList3D L, Work w);

__global__ void k_segscan(Work w);
__global__ void k_chunk_sums(Work w);

constexpr int kPostThreads = 128;   // k_chunk_sums
constexpr int kT3Threads = 256;
constexpr int kT3LocalThreads = T3_TB0 * T3_TB1;   // k_tile_local_3d: one thread per block row
constexpr int kT3LocalPerSM = 7;   // k_tile_local_3d: resident CTAs per SM (31 KB of shared memory each)
constexpr int kT3MergeThreads = 128;   // k_merge_3d threads
constexpr int kT3MergePerSM = 9;       // k_merge_3d: tiles in flight per SM (23.5 KB of shared memory each)
constexpr int kScanThreads = 256;

}  // namespace be

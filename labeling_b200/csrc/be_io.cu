// be_io.cu -- the steps either side of the labeling path, on the device: ingest (colour to gray
// and the fixed binarization of ILabeling::RGB2Gray, the slice stacking of Read3DImage) and
// egress (the colour map of LabelsToRGB and the per-plane layout of Write3DLabels).
//
// Reference (host code, OpenCV): RGB2Gray (Labeling2015/src/LabelingTools.cpp:39-49) converts a
// colour image with cv::cvtColor(COLOR_RGB2GRAY) and thresholds it at 8 to 0 / 255;
// Read3DImage (Labeling2015/main.cpp:172-212) stacks gray slices so that the slice index is the
// last (fastest) dimension of the volume; LabelsToRGB / Write3DLabels (main.cpp:248-305) colour
// labels with random colours, background black, and write the volume plane by plane along that
// last dimension.  All of it is byte shuffling bounded by HBM bandwidth: the kernels move each
// byte once, the transposes through shared-memory tiles so that both sides stay coalesced.
#include "be.h"
#include "be_api_internal.h"

#include <algorithm>
#include <cstdint>

using namespace be;

namespace {

// cv::cvtColor RGB -> gray for 8-bit data, Y = 0.299 R + 0.587 G + 0.114 B in fixed point.  OpenCV
// 3.0.0 (the version the reference builds against) rounds with 14-bit weights:
// Y = (R*4899 + G*9617 + B*1868 + 2^13) >> 14; OpenCV 4 with 15-bit weights that sum to 2^15:
// Y = (R*9798 + G*19235 + B*3735 + 2^14) >> 15 (BE_GRAY_OPENCV4).  The two differ by at most one
// gray level on some colours.
__device__ __forceinline__ uint32_t rgb_gray(uint32_t r, uint32_t g, uint32_t b, bool cv4)
{
    return cv4 ? (r * 9798u + g * 19235u + b * 3735u + (1u << 14)) >> 15
               : (r * 4899u + g * 9617u + b * 1868u + (1u << 13)) >> 14;
}

__device__ __forceinline__ uint8_t pixel_gray(const uint8_t *p, int channels, int flags)
{
    const uint32_t y = channels == 3 ? rgb_gray(p[0], p[1], p[2], (flags & BE_GRAY_OPENCV4) != 0) : p[0];
    return (flags & BE_GRAY_BINARIZE) ? (y > 8u ? 255u : 0u) : uint8_t(y);
}

__global__ void k_to_gray(const uint8_t *in, int64_t in_pitch, int channels, int rows, int cols, int flags,
                          uint8_t *out, int64_t out_pitch)
{
    const int64_t n = int64_t(rows) * cols;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t y = i / cols, x = i - y * cols;
        out[y * out_pitch + x] = pixel_gray(in + y * in_pitch + x * channels, channels, flags);
    }
}

// Slices [planes][rows][cols] (channels bytes per pixel) -> volume [rows][cols][planes].  One CTA
// per (row, 32 columns, 32 planes): loads along the columns, stores along the planes.
constexpr int TT = 32;

__global__ void __launch_bounds__(TT * 8) k_stack_slices(const uint8_t *slices, int channels, int rows, int cols,
                                                         int planes, uint8_t *vol)
{
    __shared__ uint8_t tile[TT][TT + 4];   // [plane][column]
    const int i = blockIdx.z;
    const int j0 = blockIdx.x * TT, p0 = blockIdx.y * TT;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t slice = int64_t(rows) * cols * channels;
    for (int k = ty; k < TT; k += 8) {
        const int p = p0 + k, j = j0 + tx;
        uint8_t v = 0;
        if (p < planes && j < cols) v = pixel_gray(slices + p * slice + (int64_t(i) * cols + j) * channels, channels, BE_GRAY_BINARIZE);
        tile[k][tx] = v;
    }
    __syncthreads();
    for (int k = ty; k < TT; k += 8) {
        const int j = j0 + k, p = p0 + tx;
        if (j < cols && p < planes) vol[(int64_t(i) * cols + j) * planes + p] = tile[tx][k];
    }
}

// Colour of a label: black for the background, otherwise three bytes of a 32-bit mix of
// (label, seed) (the finalizer of MurmurHash3, a published integer hash).
__device__ __forceinline__ uint32_t label_colour(int32_t l, uint32_t seed)
{
    if (l == 0) return 0u;
    uint32_t h = uint32_t(l) ^ (seed * 0x9E3779B9u);
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h & 0xFFFFFFu;
}

__global__ void k_labels_to_rgb(const int32_t *labels, int64_t n, uint32_t seed, uint8_t *rgb)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t c = label_colour(labels[i], seed);
        rgb[3 * i] = uint8_t(c);
        rgb[3 * i + 1] = uint8_t(c >> 8);
        rgb[3 * i + 2] = uint8_t(c >> 16);
    }
}

// Volume [d0][d1][d2] of labels -> d2 planes of d0 x d1 RGB pixels.  One CTA per (i, 32 j, 32 p):
// loads along the planes, stores along j.
__global__ void __launch_bounds__(TT * 8) k_volume_planes(const int32_t *labels, int d0, int d1, int d2, uint32_t seed,
                                                          uint8_t *rgb)
{
    __shared__ uint32_t tile[TT][TT + 1];   // [j][p] colours
    const int i = blockIdx.z;
    const int j0 = blockIdx.x * TT, p0 = blockIdx.y * TT;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < TT; k += 8) {
        const int j = j0 + k, p = p0 + tx;
        uint32_t c = 0;
        if (j < d1 && p < d2) c = label_colour(labels[(int64_t(i) * d1 + j) * d2 + p], seed);
        tile[k][tx] = c;
    }
    __syncthreads();
    const int64_t plane = int64_t(d0) * d1 * 3;
    for (int k = ty; k < TT; k += 8) {
        const int p = p0 + k, j = j0 + tx;
        if (p >= d2 || j >= d1) continue;
        const uint32_t c = tile[tx][k];
        uint8_t *o = rgb + p * plane + (int64_t(i) * d1 + j) * 3;
        o[0] = uint8_t(c);
        o[1] = uint8_t(c >> 8);
        o[2] = uint8_t(c >> 16);
    }
}

unsigned grid_for(be_ctx *c, int64_t n)
{
    const int64_t want = (n + 255) / 256;
    const int64_t cap = int64_t(c->sms) * 16;
    return unsigned(std::max<int64_t>(1, std::min(want, cap)));
}

int finish(be_ctx *c, const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(c, e, what);
    return BE_OK;
}

}  // namespace

extern "C" {

int be_to_gray(be_ctx *c, const uint8_t *in, int64_t in_pitch, int channels, int32_t rows, int32_t cols,
               int flags, uint8_t *out, int64_t out_pitch, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!in || !out || rows <= 0 || cols <= 0 || (channels != 1 && channels != 3) ||
        in_pitch < int64_t(cols) * channels || out_pitch < cols || (flags & ~(BE_GRAY_BINARIZE | BE_GRAY_OPENCV4)))
        return set_error(c, BE_ERR_INVALID, "be_to_gray: bad arguments");
    cudaSetDevice(c->device);
    k_to_gray<<<grid_for(c, int64_t(rows) * cols), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        in, in_pitch, channels, rows, cols, flags, out, out_pitch);
    return finish(c, "be_to_gray");
}

int be_stack_slices(be_ctx *c, const uint8_t *slices, int channels, int32_t rows, int32_t cols, int32_t planes,
                    uint8_t *volume, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!slices || !volume || rows <= 0 || cols <= 0 || planes <= 0 || rows > 65535 ||
        (channels != 1 && channels != 3))
        return set_error(c, BE_ERR_INVALID, "be_stack_slices: bad arguments");
    cudaSetDevice(c->device);
    const dim3 grid(unsigned((cols + TT - 1) / TT), unsigned((planes + TT - 1) / TT), unsigned(rows));
    k_stack_slices<<<grid, dim3(TT, 8), 0, static_cast<cudaStream_t>(stream)>>>(slices, channels, rows, cols, planes,
                                                                                volume);
    return finish(c, "be_stack_slices");
}

int be_labels_to_rgb(be_ctx *c, const int32_t *labels, int64_t n, uint32_t seed, uint8_t *rgb, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!labels || !rgb || n <= 0) return set_error(c, BE_ERR_INVALID, "be_labels_to_rgb: bad arguments");
    cudaSetDevice(c->device);
    k_labels_to_rgb<<<grid_for(c, n), 256, 0, static_cast<cudaStream_t>(stream)>>>(labels, n, seed, rgb);
    return finish(c, "be_labels_to_rgb");
}

int be_volume_to_rgb_planes(be_ctx *c, const int32_t *labels, int32_t d0, int32_t d1, int32_t d2, uint32_t seed,
                            uint8_t *rgb, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!labels || !rgb || d0 <= 0 || d1 <= 0 || d2 <= 0 || d0 > 65535)
        return set_error(c, BE_ERR_INVALID, "be_volume_to_rgb_planes: bad arguments");
    cudaSetDevice(c->device);
    const dim3 grid(unsigned((d1 + TT - 1) / TT), unsigned((d2 + TT - 1) / TT), unsigned(d0));
    k_volume_planes<<<grid, dim3(TT, 8), 0, static_cast<cudaStream_t>(stream)>>>(labels, d0, d1, d2, seed, rgb);
    return finish(c, "be_volume_to_rgb_planes");
}

}  // extern "C"

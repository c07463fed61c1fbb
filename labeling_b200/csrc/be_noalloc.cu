// be_noalloc.cu -- be_label2d_noalloc: 2D labeling that allocates no memory.
//
// Some callers cannot call cudaMalloc: a host framework that has already taken the whole device
// memory into its own pool (so a driver allocation fails or fragments that pool), a latency-bound
// loop where cudaMalloc / cudaFree would stall on an implicit device synchronization, or a plugin
// host that forbids plugins from allocating.  For them this entry point runs the same 2D
// union-find pipeline as be_label2d, but its scratch is one fixed array in the library's device
// image (`g_noalloc_scratch` below), sized for images of up to kMaxTiles tiles and kMaxSegs
// segments (4096 x 4096 pixels fit).  Every GPU that loads the library holds that array until the
// process exits.  The caller still passes its own input and output buffers.
//
// The array's name is only a stand-in in host code; the kernels receive the device address that
// cudaGetSymbolAddress returns, looked up once per device (with that device current) on the
// first call there.  All calls share the one array, so calls whose work overlaps on the GPU (other
// streams, other host threads) race: the caller must order them.  Nothing needs clearing between
// calls: every launch writes each scratch word it later reads, except the segment scan's status
// words, which carry the number of the call that wrote them (a counter in the array that each call
// increments), so words left by earlier calls are ignored; the array is zero when the library loads.
#include "be.h"
#include "be_api_internal.h"
#include "be_kernels.h"

#include <mutex>

namespace {

constexpr int64_t kMaxTiles = 1024;     // 2D tiles of 64 x 256 pixels
constexpr int64_t kMaxSegs = 65536;     // image rows x tile columns

constexpr size_t al256(size_t v) { return (v + 255) / 256 * 256; }

// Upper bound of layout_work() for kMaxTiles / kMaxSegs / one image (checked at set-up).
constexpr size_t kScratchBytes =
    al256(kMaxTiles * T2_TBW * T2_TBH * 2) +                      // block labels
    al256(kMaxTiles * T2_NPERIM * 2) +                            // border entries
    al256(kMaxTiles * (2 * T2_TBH) * (2 * T2_TBW / 32) * 4) +     // root bitmaps
    al256(kMaxTiles * 4) +                                        // node counts
    al256(kMaxTiles * T2_MAXB * 8) +                              // union-find entries
    al256(kMaxTiles * T2_MAXB * 2) +                              // root block
    al256((kMaxSegs + 15) / 16 * 16 + 16) +                       // segment counts
    al256((kMaxSegs + 1) * 4) +                                   // segment prefix
    al256(((kMaxSegs + be::kScanChunk - 1) / be::kScanChunk) * 4) +
    al256(be::kQueueWords * 4) + al256(8) + al256(64) +           // queue, count, flags
    al256(8) + al256(((kMaxSegs + be::kScanChunk - 1) / be::kScanChunk) * 8) + 4096;   // scan state, slack

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

// Device address of the scratch array on the current device, and the device's SM count (the
// launch sizes some grids by it); both looked up once per device.
int scratch_address(void **out, int *sms)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BE_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return BE_ERR_CUDA;
        if (be::layout_work(be::geometry_2d(), kMaxTiles, kMaxSegs, 1, nullptr, nullptr) > kScratchBytes)
            return BE_ERR_CUDA;
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            return BE_ERR_CUDA;
        g_sms[dev] = n;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    *sms = g_sms[dev];
    return BE_OK;
}

}  // namespace

extern "C" int be_label2d_noalloc(const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
                                  int threshold, int32_t *out, int64_t out_pitch,
                                  int64_t *n_components, void *stream)
{
    if (!in || !out || rows <= 0 || cols <= 0 || in_pitch < cols || out_pitch < cols ||
        threshold < 0 || threshold > 255)
        return BE_ERR_INVALID;
    be::Img2D im;
    be::fill_img2d(im, in, in_pitch, rows, cols, threshold, out, out_pitch, 0, 0, 0);
    const int64_t n_tiles = int64_t(im.tiles_x) * im.tiles_y;
    const int64_t n_segs = int64_t(rows) * im.tiles_x;
    if (n_tiles > kMaxTiles || n_segs > kMaxSegs) return BE_ERR_TOO_LARGE;
    void *base = nullptr;
    int sms = 0;
    int rc = scratch_address(&base, &sms);
    if (rc) return rc;
    be::Work w;
    be::layout_work(be::geometry_2d(), kMaxTiles, kMaxSegs, 1, static_cast<char *>(base), &w);
    w.n_tiles = n_tiles;
    w.n_segs = n_segs;
    w.n_chunks = int32_t((n_segs + be::kScanChunk - 1) / be::kScanChunk);
    w.n_imgs = 1;
    be::ImgList2D L{nullptr, 1, im};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (be::uf2d_launch(0, L, w, sms, false, s) != cudaSuccess) return BE_ERR_CUDA;
    if (n_components) {
        if (cudaMemcpyAsync(n_components, w.ncomp, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return BE_ERR_CUDA;
    }
    return BE_OK;
}

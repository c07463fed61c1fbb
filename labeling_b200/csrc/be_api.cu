// be_api.cu -- host side of the C ABI in include/be.h: contexts, scratch workspaces and the
// launch sequences of the 2D / 3D pipelines.
//
// The reference allocates its block buffers per call (clCreateBuffer in InitSPixels,
// LabelingAlgs.cpp:996-997 / 1451-1452) and frees them after (FreeSPixels, :1059-1063).  Here a
// context keeps one workspace per pipeline and grows it only when a larger image arrives, so a
// steady stream of calls allocates nothing.
#include "be.h"
#include "be_api_internal.h"
#include "be_kernels.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>

namespace be {

int set_error(be_ctx *ctx, int code, const char *fmt, ...)
{
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

int cuda_error(be_ctx *ctx, cudaError_t e, const char *what)
{
    return set_error(ctx, e == cudaErrorMemoryAllocation ? BE_ERR_OOM : BE_ERR_CUDA, "%s: %s (%s)",
                     what, cudaGetErrorName(e), cudaGetErrorString(e));
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// The forms that run in the iterative graph (their count and error flag live in wsiter / iter_err).
static bool iter_family(int algo) { return algo == BE_ALGO_ITER || algo == BE_ALGO_PIXEL || algo == BE_ALGO_RUNS; }

Geometry geometry_2d() { return uf2d_geometry(0); }

Geometry geometry_3d()
{
    Geometry g;
    g.lab_bytes_per_tile = size_t(T3_NBLK) * sizeof(uint32_t);
    g.rbits_bytes_per_tile = size_t(2 * T3_TB0) * (2 * T3_TB1) * (2 * T3_TB2 / 32) * sizeof(uint32_t);
    g.nperim = T3_NPERIM;
    g.maxb = T3_MAXB;
    g.links = true;
    return g;
}

// Carves the workspace of a launch with n_tiles tiles, n_segs segments and n_imgs images out of
// one allocation (or only computes its size when base == nullptr).
size_t layout_work(const Geometry &g, int64_t n_tiles, int64_t n_segs, int n_imgs, char *base, Work *w)
{
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, 256);
        return base ? base + o : nullptr;
    };
    const int64_t n_chunks = (n_segs + kScanChunk - 1) / kScanChunk;
    const size_t nodes = size_t(n_tiles) * g.maxb;
    Work t{};
    t.lab = take(size_t(n_tiles) * g.lab_bytes_per_tile);
    t.perim = reinterpret_cast<uint16_t *>(take(size_t(n_tiles) * g.nperim * sizeof(uint16_t)));
    t.rbits = reinterpret_cast<uint32_t *>(take(size_t(n_tiles) * g.rbits_bytes_per_tile));
    t.nb = reinterpret_cast<uint32_t *>(take(size_t(n_tiles) * sizeof(uint32_t)));
    t.gp = reinterpret_cast<unsigned long long *>(take(nodes * sizeof(unsigned long long)));
    t.nroot = reinterpret_cast<uint16_t *>(take(nodes * sizeof(uint16_t)));
    t.nlink = g.links ? reinterpret_cast<uint2 *>(take(nodes * sizeof(uint2))) : nullptr;
    t.segcnt = reinterpret_cast<uint8_t *>(take(align_up(size_t(n_segs), 16) + 16));
    t.segpref = reinterpret_cast<uint32_t *>(take((size_t(n_segs) + 1) * sizeof(uint32_t)));
    t.chunksum = reinterpret_cast<uint32_t *>(take(size_t(std::max<int64_t>(n_chunks, 1)) * sizeof(uint32_t)));
    t.queue = reinterpret_cast<uint32_t *>(take(kQueueWords * sizeof(uint32_t)));
    t.ncomp = reinterpret_cast<int64_t *>(take(size_t(std::max(n_imgs, 1)) * sizeof(int64_t)));
    t.err = reinterpret_cast<uint32_t *>(take(16 * sizeof(uint32_t)));
    t.epoch = reinterpret_cast<uint32_t *>(take(2 * sizeof(uint32_t)));
    t.scan_status = reinterpret_cast<uint64_t *>(take(size_t(std::max<int64_t>(n_chunks, 1)) * sizeof(uint64_t)));
    t.n_tiles = n_tiles;
    t.n_segs = n_segs;
    t.n_chunks = int32_t(n_chunks);
    t.n_imgs = n_imgs;
    if (w) *w = t;
    return off;
}

cudaError_t reset_scan_state(const Work &w, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(w.epoch, 0, 2 * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.scan_status, 0, size_t(std::max(w.n_chunks, 1)) * sizeof(uint64_t), s);
    return e;
}

int Workspace::ensure(be_ctx *ctx, const Geometry &g, int64_t n_tiles, int64_t n_segs, int n_imgs)
{
    // Node links name a segment in 32 bits.
    if (n_segs >= int64_t(kNone)) return set_error(ctx, BE_ERR_TOO_LARGE, "more than 2^32 - 2 image rows in one launch");
    const size_t need = layout_work(g, n_tiles, n_segs, n_imgs, nullptr, nullptr);
    if (!base || need > bytes) {
        if (base) {
            cudaError_t e = cudaFree(base);
            base = nullptr;
            bytes = 0;
            if (e != cudaSuccess) return cuda_error(ctx, e, "cudaFree(workspace)");
        }
        const size_t grow = need + need / 4;   // headroom for slightly larger later calls
        cudaError_t e = cudaMalloc(&base, grow);
        if (e != cudaSuccess) {
            base = nullptr;
            return cuda_error(ctx, e, "cudaMalloc(workspace)");
        }
        // The scan's status words and the launch epoch start at zero once; every later run tells
        // its own status words from older ones by the epoch it increments.
        e = cudaMemset(base, 0, grow);
        if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMemset(workspace)");
        bytes = grow;
    }
    layout_work(g, n_tiles, n_segs, n_imgs, static_cast<char *>(base), &w);
    cap_tiles = n_tiles;
    cap_segs = n_segs;
    cap_imgs = n_imgs;
    return BE_OK;
}

void Workspace::release()
{
    if (base) cudaFree(base);
    base = nullptr;
    bytes = 0;
    cap_tiles = cap_segs = 0;
    cap_imgs = 0;
}

// ---------------------------------------------------------------------------------------------
// Launch sequences.
// ---------------------------------------------------------------------------------------------
void fill_img2d(Img2D &im, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr,
                int32_t *out, int64_t out_pitch, int64_t tile_base, int64_t seg_base, int index,
                int shape)
{
    const int tbw = kShapes2D[shape].tbw, tbh = kShapes2D[shape].tbh;
    im.in = in;
    im.out = out;
    im.in_pitch = in_pitch;
    im.out_pitch = out_pitch;
    im.rows = rows;
    im.cols = cols;
    im.tiles_x = (cols + 2 * tbw - 1) / (2 * tbw);
    im.tiles_y = (rows + 2 * tbh - 1) / (2 * tbh);
    im.tile_base = tile_base;
    im.seg_base = seg_base;
    im.thr = thr;
    im.index = index;
}

void fill_img3d(Img3D &im, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int thr,
                int32_t *out, int64_t tile_base, int64_t seg_base, int index)
{
    im.in = in;
    im.out = out;
    im.d0 = d0;
    im.d1 = d1;
    im.d2 = d2;
    im.t0 = (d0 + 2 * T3_TB0 - 1) / (2 * T3_TB0);
    im.t1 = (d1 + 2 * T3_TB1 - 1) / (2 * T3_TB1);
    im.t2 = (d2 + 2 * T3_TB2 - 1) / (2 * T3_TB2);
    im.tile_base = tile_base;
    im.seg_base = seg_base;
    im.thr = thr;
    im.index = index;
}

cudaError_t launch_uf3d(const ImgList3D &L, const Work &w, int sms, bool persistent, cudaStream_t s,
                        cudaEvent_t *ev)
{
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], s);
    };
    auto grid = [&](int64_t items, int per_sm) -> unsigned {
        int64_t g = persistent ? std::min<int64_t>(items, int64_t(sms) * per_sm) : items;
        return unsigned(std::max<int64_t>(g, 1));
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
    k_tile_local_3d<<<grid(w.n_tiles, kT3LocalPerSM), kT3LocalThreads, 0, s>>>(L, wk);
    keep(cudaGetLastError());
    mark(1);
    keep(launch_k(k_merge_3d, grid(w.n_tiles, kT3MergePerSM), kT3MergeThreads, s, ov, L, wk));
    mark(2);
    keep(launch_k(k_scan_link_3d, grid(int64_t(w.n_chunks) + w.n_tiles, 8), kScanThreads, s, ov, L, wk));
    mark(3);
    // The label writes run a fixed tile order over 5 CTAs per SM (they prefetch their next tile).
    keep(launch_k(k_tile_write_3d, unsigned(std::max<int64_t>(1, std::min<int64_t>(w.n_tiles, int64_t(sms) * 5))),
                  kT3Threads, s, ov, L, wk));
    mark(4);
    return e;
}

}  // namespace be

using namespace be;

// ---------------------------------------------------------------------------------------------
// C ABI.
// ---------------------------------------------------------------------------------------------
extern "C" {

const char *be_version(void) { return "0.1.0"; }

int be_create(be_ctx **out, int device)
{
    if (!out) return BE_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return BE_ERR_CUDA;
    if (device < 0 || device >= ndev) return BE_ERR_INVALID;
    be_ctx *c = new be_ctx();
    c->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_ncomp, 64 * sizeof(int64_t));
    for (int i = 0; i <= kStages && e == cudaSuccess; ++i) e = cudaEventCreate(&c->stage_ev[i]);
    if (e != cudaSuccess) {
        be_destroy(c);
        return e == cudaErrorMemoryAllocation ? BE_ERR_OOM : BE_ERR_CUDA;
    }
    *out = c;
    return BE_OK;
}

int be_destroy(be_ctx *c)
{
    if (!c) return BE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->ws2d.release();
    c->ws3d.release();
    c->wsiter.release();
    for (be_iter_graph &g : c->iter_graph) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    if (c->d_in) cudaFree(c->d_in);
    if (c->d_out) cudaFree(c->d_out);
    if (c->slab_buf) cudaFree(c->slab_buf);
    if (c->h_ncomp) cudaFreeHost(c->h_ncomp);
    for (int i = 0; i <= kStages; ++i)
        if (c->stage_ev[i]) cudaEventDestroy(c->stage_ev[i]);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return BE_OK;
}

const char *be_last_error(const be_ctx *c) { return c ? c->err.c_str() : "no context"; }

int be_check_status(be_ctx *c, int dims, uint32_t *out3)
{
    if (!c || !out3 || (dims != 2 && dims != 3)) return BE_ERR_INVALID;
    out3[0] = out3[1] = out3[2] = 0;
    const Work &w = dims == 2 ? c->ws2d.w : c->ws3d.w;
    if (!w.err) return BE_OK;
    cudaError_t e = cudaMemcpy(out3, w.err, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(c, e, "be_check_status");
    return BE_OK;
}

int be_set_stage_timing(be_ctx *c, int enable)
{
    if (!c) return BE_ERR_INVALID;
    c->timing = enable != 0;
    c->timed_stages = 0;
    return BE_OK;
}

int be_stage_times(be_ctx *c, float *ms, int max_stages, int *n_stages)
{
    if (!c || !n_stages) return BE_ERR_INVALID;
    *n_stages = c->timed_stages;
    if (!c->timed_stages) return BE_OK;
    cudaError_t e = cudaEventSynchronize(c->stage_ev[c->timed_stages]);
    if (e != cudaSuccess) return cuda_error(c, e, "be_stage_times");
    for (int i = 0; i < c->timed_stages && i < max_stages; ++i) {
        e = cudaEventElapsedTime(&ms[i], c->stage_ev[i], c->stage_ev[i + 1]);
        if (e != cudaSuccess) return cuda_error(c, e, "be_stage_times");
    }
    return BE_OK;
}

int be_label2d(be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
               int threshold, int coh, int algo, int32_t *out, int64_t out_pitch,
               int64_t *n_components, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!in || !out) return set_error(c, BE_ERR_INVALID, "be_label2d: null buffer");
    if (rows <= 0 || cols <= 0 || int64_t(rows) * cols >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "be_label2d: bad size %d x %d", rows, cols);
    if (in_pitch < cols || out_pitch < cols)
        return set_error(c, BE_ERR_INVALID, "be_label2d: pitch smaller than the row");
    if (threshold < 0 || threshold > 255)
        return set_error(c, BE_ERR_INVALID, "be_label2d: threshold %d outside 0..255", threshold);
    if (algo < BE_ALGO_AUTO || algo > BE_ALGO_RUNS)
        return set_error(c, BE_ERR_INVALID, "be_label2d: unknown algorithm %d", algo);
    if (coh == BE_COH_4 && algo != BE_ALGO_PIXEL && algo != BE_ALGO_RUNS)
        return set_error(c, BE_ERR_INVALID, "be_label2d: block equivalence does not support 4-connectivity");
    if (coh != BE_COH_4 && coh != BE_COH_8 && coh != BE_COH_DEFAULT)
        return set_error(c, BE_ERR_INVALID, "be_label2d: unknown connectivity %d", coh);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaSetDevice");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc, shape;
    pick2d(c, rows, cols, algo, &algo, &shape);
    c->last_algo = algo;
    if (algo == BE_ALGO_PIXEL) {
        rc = run_lbeq2d(c, in, in_pitch, rows, cols, threshold, coh == BE_COH_8, out, out_pitch, s);
    } else if (algo == BE_ALGO_RUNS) {
        rc = run_runeq2d(c, in, in_pitch, rows, cols, threshold, coh == BE_COH_8, out, out_pitch, s);
    } else if (algo == BE_ALGO_ITER) {
        rc = run_iter2d(c, in, in_pitch, rows, cols, threshold, out, out_pitch, s);
    } else {
        Img2D im;
        fill_img2d(im, in, in_pitch, rows, cols, threshold, out, out_pitch, 0, 0, 0, shape);
        const int64_t n_tiles = int64_t(im.tiles_x) * im.tiles_y;
        const int64_t n_segs = int64_t(rows) * im.tiles_x;
        rc = c->ws2d.ensure(c, uf2d_geometry(shape), n_tiles, n_segs, 1);
        if (rc) return rc;
        ImgList2D L{nullptr, 1, im};
#ifdef BE_BOUNDS_CHECK
        cudaMemsetAsync(c->ws2d.w.err, 0, 16 * sizeof(uint32_t), s);
#endif
        e = uf2d_launch(shape, L, c->ws2d.w, c->sms, false, s, c->timing ? c->stage_ev : nullptr);
        c->timed_stages = c->timing ? kStages2D : 0;
        if (e != cudaSuccess) return cuda_error(c, e, "be_label2d launch");
    }
    if (rc) return rc;
    if (n_components) {
        const int64_t *src = iter_family(algo) ? c->wsiter.w.ncomp : c->ws2d.w.ncomp;
        e = cudaMemcpyAsync(c->h_ncomp, src, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_error(c, e, "be_label2d sync");
        if (iter_family(algo) && c->iter_err && *c->iter_err)
            return set_error(c, BE_ERR_NO_CONVERGENCE, "be_label2d: iteration cap reached");
        *n_components = c->h_ncomp[0];
    }
    return BE_OK;
}

int be_label3d(be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int threshold,
               int algo, int32_t *out, int64_t *n_components, void *stream)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!in || !out) return set_error(c, BE_ERR_INVALID, "be_label3d: null buffer");
    if (d0 <= 0 || d1 <= 0 || d2 <= 0 || int64_t(d0) * d1 * d2 >= (int64_t(1) << 31))
        return set_error(c, BE_ERR_INVALID, "be_label3d: bad size %d x %d x %d", d0, d1, d2);
    if (threshold < 0 || threshold > 255)
        return set_error(c, BE_ERR_INVALID, "be_label3d: threshold %d outside 0..255", threshold);
    if (algo < BE_ALGO_AUTO || algo > BE_ALGO_PIXEL)
        return set_error(c, BE_ERR_INVALID, algo == BE_ALGO_RUNS ? "be_label3d: run equivalence is 2D only"
                                                                 : "be_label3d: unknown algorithm %d", algo);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaSetDevice");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    pick3d(c, int64_t(d0) * d1 * d2, algo, &algo);
    c->last_algo = algo;
    if (algo == BE_ALGO_PIXEL) {
        rc = run_lbeq3d(c, in, d0, d1, d2, threshold, out, s);
    } else if (algo == BE_ALGO_ITER) {
        rc = run_iter3d(c, in, d0, d1, d2, threshold, out, s);
    } else {
        Img3D im;
        fill_img3d(im, in, d0, d1, d2, threshold, out, 0, 0, 0);
        const int64_t n_tiles = int64_t(im.t0) * im.t1 * im.t2;
        const int64_t n_segs = int64_t(d0) * d1 * im.t2;
        rc = c->ws3d.ensure(c, geometry_3d(), n_tiles, n_segs, 1);
        if (rc) return rc;
        ImgList3D L{nullptr, 1, im};
#ifdef BE_BOUNDS_CHECK
        cudaMemsetAsync(c->ws3d.w.err, 0, 16 * sizeof(uint32_t), s);
#endif
        e = launch_uf3d(L, c->ws3d.w, c->sms, false, s, c->timing ? c->stage_ev : nullptr);
        c->timed_stages = c->timing ? kStages3D : 0;
        if (e != cudaSuccess) return cuda_error(c, e, "be_label3d launch");
    }
    if (rc) return rc;
    if (n_components) {
        const int64_t *src = iter_family(algo) ? c->wsiter.w.ncomp : c->ws3d.w.ncomp;
        e = cudaMemcpyAsync(c->h_ncomp, src, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_error(c, e, "be_label3d sync");
        if (iter_family(algo) && c->iter_err && *c->iter_err)
            return set_error(c, BE_ERR_NO_CONVERGENCE, "be_label3d: iteration cap reached");
        *n_components = c->h_ncomp[0];
    }
    return BE_OK;
}

static int ensure_staging(be_ctx *c, size_t in_bytes, size_t out_bytes)
{
    cudaError_t e;
    if (in_bytes > c->d_in_bytes) {
        if (c->d_in) cudaFree(c->d_in);
        c->d_in = nullptr;
        c->d_in_bytes = 0;
        e = cudaMalloc(&c->d_in, in_bytes);
        if (e != cudaSuccess) return cuda_error(c, e, "cudaMalloc(input staging)");
        c->d_in_bytes = in_bytes;
    }
    if (out_bytes > c->d_out_bytes) {
        if (c->d_out) cudaFree(c->d_out);
        c->d_out = nullptr;
        c->d_out_bytes = 0;
        e = cudaMalloc(&c->d_out, out_bytes);
        if (e != cudaSuccess) return cuda_error(c, e, "cudaMalloc(output staging)");
        c->d_out_bytes = out_bytes;
    }
    return BE_OK;
}

int be_label2d_host(be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
                    int threshold, int coh, int algo, int32_t *out, int64_t out_pitch,
                    int64_t *n_components, double *elapsed_us)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!in || !out) return set_error(c, BE_ERR_INVALID, "be_label2d_host: null buffer");
    if (rows <= 0 || cols <= 0 || in_pitch < cols || out_pitch < cols)
        return set_error(c, BE_ERR_INVALID, "be_label2d_host: bad size or pitch");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaSetDevice");
    const int64_t dpi = (int64_t(cols) + 15) / 16 * 16, dpo = (int64_t(cols) + 3) / 4 * 4;
    int rc = ensure_staging(c, size_t(dpi) * rows, size_t(dpo) * rows * sizeof(int32_t));
    if (rc) return rc;
    cudaStream_t s = c->stream;
    e = cudaMemcpy2DAsync(c->d_in, dpi, in, in_pitch, cols, rows, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_error(c, e, "upload");
    cudaEventRecord(c->ev0, s);
    int64_t n = 0;
    rc = be_label2d(c, static_cast<const uint8_t *>(c->d_in), dpi, rows, cols, threshold, coh, algo,
                    static_cast<int32_t *>(c->d_out), dpo, nullptr, s);
    if (rc) return rc;
    cudaEventRecord(c->ev1, s);
    e = cudaMemcpy2DAsync(out, out_pitch * sizeof(int32_t), c->d_out, dpo * sizeof(int32_t),
                          cols * sizeof(int32_t), rows, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_error(c, e, "download");
    const int64_t *src = iter_family(c->last_algo) ? c->wsiter.w.ncomp : c->ws2d.w.ncomp;
    e = cudaMemcpyAsync(c->h_ncomp, src, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(c, e, "be_label2d_host sync");
    if (iter_family(c->last_algo) && c->iter_err && *c->iter_err)
        return set_error(c, BE_ERR_NO_CONVERGENCE, "be_label2d_host: iteration cap reached");
    n = c->h_ncomp[0];
    if (n_components) *n_components = n;
    if (elapsed_us) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        *elapsed_us = double(ms) * 1000.0;
    }
    return BE_OK;
}

int be_label3d_host(be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2,
                    int threshold, int algo, int32_t *out, int64_t *n_components,
                    double *elapsed_us)
{
    if (!c) return BE_ERR_INVALID;
    c->err.clear();
    if (!in || !out) return set_error(c, BE_ERR_INVALID, "be_label3d_host: null buffer");
    if (d0 <= 0 || d1 <= 0 || d2 <= 0)
        return set_error(c, BE_ERR_INVALID, "be_label3d_host: bad size");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_error(c, e, "cudaSetDevice");
    const size_t n = size_t(d0) * d1 * d2;
    int rc = ensure_staging(c, n, n * sizeof(int32_t));
    if (rc) return rc;
    cudaStream_t s = c->stream;
    e = cudaMemcpyAsync(c->d_in, in, n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_error(c, e, "upload");
    cudaEventRecord(c->ev0, s);
    rc = be_label3d(c, static_cast<const uint8_t *>(c->d_in), d0, d1, d2, threshold, algo,
                    static_cast<int32_t *>(c->d_out), nullptr, s);
    if (rc) return rc;
    cudaEventRecord(c->ev1, s);
    e = cudaMemcpyAsync(out, c->d_out, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_error(c, e, "download");
    const int64_t *src = iter_family(c->last_algo) ? c->wsiter.w.ncomp : c->ws3d.w.ncomp;
    e = cudaMemcpyAsync(c->h_ncomp, src, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(c, e, "be_label3d_host sync");
    if (iter_family(c->last_algo) && c->iter_err && *c->iter_err)
        return set_error(c, BE_ERR_NO_CONVERGENCE, "be_label3d_host: iteration cap reached");
    if (n_components) *n_components = c->h_ncomp[0];
    if (elapsed_us) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        *elapsed_us = double(ms) * 1000.0;
    }
    return BE_OK;
}

}  // extern "C"

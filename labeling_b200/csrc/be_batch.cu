// be_batch.cu -- batched labeling: a list of 2D images and 3D volumes of any sizes labeled by ONE
// launch sequence captured in a CUDA graph.
//
// The reference labels one image per call with a host loop in between
// (ProcessImages, main.cpp:309-340).  Here the images of a batch share one workspace and one
// descriptor array; every kernel of the union-find pipeline runs persistent CTAs (SMs x resident
// blocks) that pull tiles -- not images -- from an atomic work queue, so thousands of uneven
// images balance by tiles.  The 2D chain and the 3D chain are two branches of the same graph.
// be_batch_tune times the 2D tile shapes and the persistent / one-CTA-per-tile choice on the
// batch itself and keeps the fastest graph.
#include "be.h"
#include "be_api_internal.h"
#include "be_kernels.h"

#include <algorithm>
#include <vector>

using namespace be;

struct be_batch {
    be_ctx *ctx = nullptr;
    int n = 0;
    std::vector<be_image> imgs;
    std::vector<int> idx2d, idx3d;   // positions in the caller's list
    int shape = 0;                   // 2D tile shape
    bool persistent = true;
    void *dev = nullptr;             // descriptors + workspaces + counts
    size_t dev_bytes = 0;
    int64_t *counts = nullptr;       // per image, in caller order
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr, cap2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

namespace {

size_t al256(size_t v) { return (v + 255) / 256 * 256; }

void release_graph(be_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// (Re)builds descriptors, workspaces and the graph for the current shape / persistence.
int build(be_batch *b)
{
    be_ctx *c = b->ctx;
    release_graph(b);
    if (b->dev) cudaFree(b->dev);
    b->dev = nullptr;

    std::vector<Img2D> d2(b->idx2d.size());
    std::vector<Img3D> d3(b->idx3d.size());
    int64_t t2 = 0, s2 = 0, t3 = 0, s3 = 0;
    for (size_t i = 0; i < b->idx2d.size(); ++i) {
        const be_image &im = b->imgs[b->idx2d[i]];
        fill_img2d(d2[i], im.in, im.in_pitch, im.dims[0], im.dims[1], im.threshold, im.out,
                   im.out_pitch, t2, s2, b->idx2d[i], b->shape);
        t2 += int64_t(d2[i].tiles_x) * d2[i].tiles_y;
        s2 += int64_t(im.dims[0]) * d2[i].tiles_x;
    }
    for (size_t i = 0; i < b->idx3d.size(); ++i) {
        const be_image &im = b->imgs[b->idx3d[i]];
        fill_img3d(d3[i], im.in, im.dims[0], im.dims[1], im.dims[2], im.threshold, im.out, t3, s3,
                   b->idx3d[i]);
        t3 += int64_t(d3[i].t0) * d3[i].t1 * d3[i].t2;
        s3 += int64_t(im.dims[0]) * im.dims[1] * d3[i].t2;
    }
    const Geometry g2 = uf2d_geometry(b->shape), g3 = geometry_3d();
    const size_t w2 = d2.empty() ? 0 : layout_work(g2, t2, s2, b->n, nullptr, nullptr);
    const size_t w3 = d3.empty() ? 0 : layout_work(g3, t3, s3, b->n, nullptr, nullptr);
    const size_t o_d2 = 0, o_d3 = al256(d2.size() * sizeof(Img2D));
    const size_t o_cnt = o_d3 + al256(d3.size() * sizeof(Img3D));
    const size_t o_w2 = o_cnt + al256(size_t(b->n) * sizeof(int64_t));
    const size_t o_w3 = o_w2 + al256(w2);
    const size_t total = o_w3 + al256(w3);
    cudaError_t e = cudaMalloc(&b->dev, total);
    if (e != cudaSuccess) {
        b->dev = nullptr;
        return cuda_error(c, e, "be_batch: cudaMalloc");
    }
    b->dev_bytes = total;
    e = cudaMemset(b->dev, 0, total);   // scan status words and launch epochs start at zero
    if (e != cudaSuccess) return cuda_error(c, e, "be_batch: cudaMemset");
    char *base = static_cast<char *>(b->dev);
    b->counts = reinterpret_cast<int64_t *>(base + o_cnt);
    if (!d2.empty()) e = cudaMemcpy(base + o_d2, d2.data(), d2.size() * sizeof(Img2D), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !d3.empty())
        e = cudaMemcpy(base + o_d3, d3.data(), d3.size() * sizeof(Img3D), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(c, e, "be_batch: descriptor upload");
    Work W2{}, W3{};
    if (!d2.empty()) {
        layout_work(g2, t2, s2, b->n, base + o_w2, &W2);
        W2.ncomp = b->counts;
    }
    if (!d3.empty()) {
        layout_work(g3, t3, s3, b->n, base + o_w3, &W3);
        W3.ncomp = b->counts;
    }
    ImgList2D L2{reinterpret_cast<const Img2D *>(base + o_d2), int(d2.size()), d2.empty() ? Img2D{} : d2[0]};
    ImgList3D L3{reinterpret_cast<const Img3D *>(base + o_d3), int(d3.size()), d3.empty() ? Img3D{} : d3[0]};

    // Capture: the 2D chain on `cap`, the 3D chain forked onto `cap2`.
    e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_error(c, e, "be_batch: begin capture");
    cudaError_t le = cudaSuccess;
    if (!d3.empty()) {
        cudaEventRecord(b->fork, b->cap);
        cudaStreamWaitEvent(b->cap2, b->fork, 0);
        if (b->persistent) cudaMemsetAsync(W3.queue, 0, kQueueWords * sizeof(uint32_t), b->cap2);
        le = launch_uf3d(L3, W3, c->sms, b->persistent, b->cap2);
        cudaEventRecord(b->join, b->cap2);
    }
    if (!d2.empty() && le == cudaSuccess) {
        if (b->persistent) cudaMemsetAsync(W2.queue, 0, kQueueWords * sizeof(uint32_t), b->cap);
        le = uf2d_launch(b->shape, L2, W2, c->sms, b->persistent, b->cap);
    }
    if (!d3.empty()) cudaStreamWaitEvent(b->cap, b->join, 0);
    e = cudaStreamEndCapture(b->cap, &b->graph);
    if (le != cudaSuccess) return cuda_error(c, le, "be_batch: capture launch");
    if (e != cudaSuccess) return cuda_error(c, e, "be_batch: end capture");
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return cuda_error(c, e, "be_batch: instantiate");
    return BE_OK;
}

}  // namespace

extern "C" {

int be_batch_create(be_ctx *c, const be_image *imgs, int n, int flags, be_batch **out)
{
    if (!c || !imgs || n <= 0 || !out) return BE_ERR_INVALID;
    *out = nullptr;
    c->err.clear();
    be_batch *b = new be_batch();
    b->ctx = c;
    b->n = n;
    b->imgs.assign(imgs, imgs + n);
    b->persistent = !(flags & BE_BATCH_ONE_CTA_PER_TILE);
    for (int i = 0; i < n; ++i) {
        const be_image &im = imgs[i];
        const bool is3d = im.dims[2] > 0;
        const int64_t vol = int64_t(im.dims[0]) * im.dims[1] * (is3d ? im.dims[2] : 1);
        if (!im.in || !im.out || im.dims[0] <= 0 || im.dims[1] <= 0 || vol >= (int64_t(1) << 31) ||
            im.threshold < 0 || im.threshold > 255 ||
            (!is3d && (im.in_pitch < im.dims[1] || im.out_pitch < im.dims[1]))) {
            delete b;
            return set_error(c, BE_ERR_INVALID, "be_batch_create: bad image %d", i);
        }
        (is3d ? b->idx3d : b->idx2d).push_back(i);
    }
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        be_batch_destroy(b);
        return cuda_error(c, e, "be_batch_create");
    }
    int rc = build(b);
    if (rc) {
        be_batch_destroy(b);
        return rc;
    }
    *out = b;
    return BE_OK;
}

int be_batch_run(be_batch *b, void *stream)
{
    if (!b || !b->exec) return BE_ERR_INVALID;
    cudaError_t e = cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_error(b->ctx, e, "be_batch_run");
    return BE_OK;
}

int be_batch_counts(be_batch *b, int64_t *counts, void *stream)
{
    if (!b || !counts) return BE_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(counts, b->counts, size_t(b->n) * sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(b->ctx, e, "be_batch_counts");
    return BE_OK;
}

int be_batch_tune(be_batch *b, void *stream, int *choice)
{
    if (!b) return BE_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int best_shape = b->shape;
    bool best_pers = b->persistent;
    const int nshape = b->idx2d.empty() ? 1 : kNumShapes2D;
    for (int pers = 1; pers >= 0; --pers) {
        for (int sh = 0; sh < nshape; ++sh) {
            b->shape = sh;
            b->persistent = pers != 0;
            int rc = build(b);
            if (rc) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return rc;
            }
            float ms = 0;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(e0, s);
                cudaGraphLaunch(b->exec, s);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float t = 0;
                cudaEventElapsedTime(&t, e0, e1);
                if (rep) ms += t;
            }
            if (ms < best) {
                best = ms;
                best_shape = sh;
                best_pers = pers != 0;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->shape = best_shape;
    b->persistent = best_pers;
    int rc = build(b);
    if (choice) *choice = best_shape | (best_pers ? 0 : BE_BATCH_ONE_CTA_PER_TILE);
    return rc;
}

int be_batch_destroy(be_batch *b)
{
    if (!b) return BE_OK;
    if (b->ctx) cudaSetDevice(b->ctx->device);
    if (b->cap) cudaStreamSynchronize(b->cap);
    release_graph(b);
    if (b->dev) cudaFree(b->dev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->cap2) cudaStreamDestroy(b->cap2);
    delete b;
    return BE_OK;
}

}  // extern "C"

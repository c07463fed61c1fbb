// be_api_internal.h -- host-side state behind the C ABI (not part of the public interface).
#pragma once
#include "be.h"
#include "be_common.cuh"

#include <cuda_runtime.h>
#include <string>
#include <vector>

namespace be {

constexpr int kQueueWords = 16;   // work-queue counters per workspace (one per kernel)

// Per-tile sizes of a pipeline's workspace.
struct Geometry {
    size_t lab_bytes_per_tile;
    size_t rbits_bytes_per_tile;
    int nperim;
    int maxb;
    bool links = false;   // the pipeline resolves node links (Work::nlink) before its label writes
};

// 2D tile shapes (in 2x2 blocks); shape 0 is the default.
struct Shape2D {
    int tbw, tbh;
};
constexpr int kNumShapes2D = 3;
extern const Shape2D kShapes2D[kNumShapes2D];
Geometry uf2d_geometry(int shape);
cudaError_t uf2d_launch(int shape, const ImgList2D &L, const Work &w, int sms, bool persistent,
                        cudaStream_t s, cudaEvent_t *ev = nullptr);

Geometry geometry_2d();   // shape 0
Geometry geometry_3d();
size_t layout_work(const Geometry &g, int64_t n_tiles, int64_t n_segs, int n_imgs, char *base, Work *w);
// Zeroes a workspace's launch epoch and scan status words (memory that was not zeroed before).
cudaError_t reset_scan_state(const Work &w, cudaStream_t s);

// One growable device allocation holding a Work.
struct Workspace {
    void *base = nullptr;
    size_t bytes = 0;
    int64_t cap_tiles = 0, cap_segs = 0;
    int cap_imgs = 0;
    Work w{};
    int ensure(struct ::be_ctx *ctx, const Geometry &g, int64_t n_tiles, int64_t n_segs, int n_imgs);
    void release();
};

// Scratch of the iterative (scan / analyze) form.
struct IterWork {
    void *base = nullptr;
    size_t bytes = 0;
};

// One autotuner decision: size class -> algorithm (+ 2D tile shape), with the time it measured.
struct TuneEntry {
    uint32_t cls;
    int algo;
    int shape;
    float us;
};
void pick2d(const struct ::be_ctx *c, int rows, int cols, int algo_in, int *algo, int *shape);
void pick3d(const struct ::be_ctx *c, int64_t n, int algo_in, int *algo);

int set_error(struct ::be_ctx *ctx, int code, const char *fmt, ...);
int cuda_error(struct ::be_ctx *ctx, cudaError_t e, const char *what);

void fill_img2d(Img2D &im, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr,
                int32_t *out, int64_t out_pitch, int64_t tile_base, int64_t seg_base, int index,
                int shape = 0);
void fill_img3d(Img3D &im, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int thr,
                int32_t *out, int64_t tile_base, int64_t seg_base, int index);
constexpr int kStages = 5;     // stage events a context keeps (at least the launches of a pipeline)
constexpr int kStages2D = 4;   // launches of the 2D union-find pipeline
constexpr int kStages3D = 4;   // launches of the 3D union-find pipeline
cudaError_t launch_uf3d(const ImgList3D &L, const Work &w, int sms, bool persistent, cudaStream_t s,
                        cudaEvent_t *ev = nullptr);

int run_iter2d(struct ::be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
               int thr, int32_t *out, int64_t out_pitch, cudaStream_t s);
int run_iter3d(struct ::be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int thr,
               int32_t *out, cudaStream_t s);
int run_lbeq2d(struct ::be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr,
               int conn8, int32_t *out, int64_t out_pitch, cudaStream_t s);
int run_lbeq3d(struct ::be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int thr,
               int32_t *out, cudaStream_t s);
int run_runeq2d(struct ::be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int thr,
                int conn8, int32_t *out, int64_t out_pitch, cudaStream_t s);

}  // namespace be

// An instantiated graph of the iterative form, kept for the next call of the same form and sizes.
struct be_iter_graph {
    std::vector<unsigned char> key;   // the graph's baked-in arguments, image buffers blanked
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t init = nullptr, fin = nullptr;   // the nodes that read / write the image
};

struct be_ctx {
    int device = 0;
    int sms = 148;
    std::string err;
    be::Workspace ws2d, ws3d, wsiter;
    void *iter_base = nullptr;      // iterative-form block arrays
    size_t iter_bytes = 0;
    uint32_t *iter_err = nullptr;   // pinned: iteration-cap flag of the last iterative call
    void *d_in = nullptr, *d_out = nullptr;   // device staging of the *_host calls
    size_t d_in_bytes = 0, d_out_bytes = 0;
    void *slab_buf = nullptr;       // be_slab_relabel: label map + joined lists
    size_t slab_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t *h_ncomp = nullptr;     // pinned
    bool timing = false;            // record an event between the launches of a plain call
    int timed_stages = 0;
    cudaEvent_t stage_ev[be::kStages + 1] = {};
    std::vector<be::TuneEntry> tune;  // autotuner decisions
    int last_algo = 1;                // algorithm the last label call actually ran
    be_iter_graph iter_graph[5];      // iterative form: 2D / 3D blocks, 2D / 3D pixels, 2D runs
};

/*
 * be.h -- C ABI of the B200 Block-Equivalence (BE) connected-component labeler.
 *
 * Plain C: pointers, sizes and int status codes only.  Every entry point returns BE_OK (0) or a
 * positive be_status; be_last_error() gives the message of the last failure on a context.
 *
 * Labels.  Output labels are int32, 0 = background, components numbered 1..K in the order of
 * their first foreground pixel (voxel) in raster order (row-major; for volumes the last dimension
 * is the fastest).  This is the reference BE result after canonical relabeling: the reference's
 * own label values (1 + smallest block index in its padded block grid) differ only by a
 * renumbering.  Foreground is `pixel > threshold`; threshold 0 reproduces the reference kernels'
 * `pixel != 0` test and threshold 8 the binarization of ILabeling::RGB2Gray
 * (Labeling2015/src/LabelingTools.cpp:39-49).
 *
 * Connectivity.  2D: 8-connectivity with 2x2 blocks (reference LBEQ2_*, LabelingAlgs.cl:136-319).
 * 3D: 26-connectivity with 2x2x2 blocks (reference BLEQ3D_*, LabelingAlgs.cl:740-979).
 *
 * Threading.  A context is used by one host thread at a time.  Device buffers are owned by the
 * caller; the context owns and reuses its scratch.  `stream` is a cudaStream_t (NULL = the legacy
 * default stream).  Calls return once the work is enqueued, except where a host result is asked
 * for (n_components != NULL, the *_host variants), which synchronize the stream.
 */
#ifndef BE_B200_H_
#define BE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum be_status {
    BE_OK = 0,
    BE_ERR_INVALID = 1,        /* bad argument (null pointer, size, pitch, unsupported mode) */
    BE_ERR_OOM = 2,            /* device or pinned host allocation failed */
    BE_ERR_NO_CONVERGENCE = 3, /* iterative merge hit its iteration cap */
    BE_ERR_CUDA = 4,           /* a CUDA call failed; see be_last_error */
    BE_ERR_TIMEOUT = 5,        /* a bounded wait ran out (server / batch) */
    BE_ERR_BUSY = 6,           /* admission refused: not enough free device memory or slots */
    BE_ERR_CANCELLED = 7,      /* the request was cancelled before it completed */
    BE_ERR_TOO_LARGE = 8       /* the image exceeds the fixed scratch of be_label2d_noalloc, or one
                                  launch holds more than 2^32 - 2 image rows (voxel rows) */
} be_status;

/* Merge algorithm. */
enum {
    BE_ALGO_AUTO = 0, /* the autotuned choice (union-find unless the tuner measured otherwise) */
    BE_ALGO_UF = 1,   /* tile union-find in shared memory + global border merge */
    BE_ALGO_ITER = 2, /* the paper's iterative scan / analyze, with a device-side change flag */
    BE_ALGO_PIXEL = 3, /* pixel-level label equivalence, the -a lbeq path (LabelingAlgs.cl:31-130,
                          635-734): 2D 4-connectivity for BE_COH_4 / BE_COH_DEFAULT (the reference's
                          default), 8 for BE_COH_8; 3D 26-connectivity */
    BE_ALGO_RUNS = 4   /* 2D run equivalence, the -a runeq -g path (TOCLRunEquivLabeling,
                          LabelingAlgs.cpp:1090-1268, RE* kernels LabelingAlgs.cl:325-616): runs of
                          each row joined by column overlap -- 4-connectivity for BE_COH_4 /
                          BE_COH_DEFAULT (the reference's runs), 8 for BE_COH_8; 2D only */
};

/* Connectivity selector, as the reference's TCoherence (LabelingTools.hpp:45-50). */
enum { BE_COH_4 = 0, BE_COH_8 = 1, BE_COH_DEFAULT = 2 };

typedef struct be_ctx be_ctx;

/* Library version string ("major.minor.patch"). */
const char *be_version(void);

/* Context on CUDA device `device`.  Replaces IOCLLabeling::Init / InitOpenCL
 * (LabelingTools.cpp:81-94, CLUtils.c:88-233): no runtime compilation, kernels are built in. */
int be_create(be_ctx **ctx, int device);
int be_destroy(be_ctx *ctx);
/* Message of the last failed call on ctx (empty string when none). */
const char *be_last_error(const be_ctx *ctx);

/* 2D labeling of a device image.  Replaces TOCLLabelEquivalenceX2::DoOCLLabel
 * (LabelingAlgs.cpp:1067-1084, kernels LabelingAlgs.cl:176-319) minus its padding: any
 * rows x cols works, rows >= 1, cols >= 1, rows * cols < 2^31.
 *   in       uint8 pixels, in_pitch bytes per row (>= cols)
 *   out      int32 labels, out_pitch elements per row (>= cols); every pixel is written
 *   coh      BE_COH_8 or BE_COH_DEFAULT (8-connectivity); BE_COH_4 is rejected like the
 *            reference (LabelingAlgs.cpp:1070)
 *   n_components  if not NULL: receives K (synchronizes `stream`)
 */
int be_label2d(be_ctx *ctx, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
               int threshold, int coh, int algo, int32_t *out, int64_t out_pitch,
               int64_t *n_components, void *stream);

/* 3D labeling of a dense device volume [d0][d1][d2] (d2 fastest).  Replaces
 * TOCLBlockEquivalence3D::DoOCLLabel3D (LabelingAlgs.cpp:1520-1536, kernels
 * LabelingAlgs.cl:805-979) minus the padding; d0 * d1 * d2 < 2^31.  Output is the unpadded
 * volume (the reference returns its padded copy, LabelingTools.cpp:217-220). */
int be_label3d(be_ctx *ctx, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int threshold,
               int algo, int32_t *out, int64_t *n_components, void *stream);

/* Host-buffer variants: copy in through pinned staging, label, copy out, synchronize.  The
 * equivalent of IOCLLabeling::Label / IOCLLabeling3D::Label (LabelingTools.cpp:98-132, 180-221)
 * around the device call.  elapsed_us (optional) receives the device time of the labeling alone,
 * measured with CUDA events (the reference's watch_ scope). */
int be_label2d_host(be_ctx *ctx, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
                    int threshold, int coh, int algo, int32_t *out, int64_t out_pitch,
                    int64_t *n_components, double *elapsed_us);
int be_label3d_host(be_ctx *ctx, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2,
                    int threshold, int algo, int32_t *out, int64_t *n_components,
                    double *elapsed_us);

/* ---- Autotuner (no counterpart in the reference) ----------------------------------------------
 * Times the candidate forms -- the union-find pipeline in each 2D tile shape (32x128, 64x64,
 * 16x256 blocks) and the iterative scan/analyze form -- on the caller's own input, checks that all
 * of them give identical labels, and remembers the fastest for the input's size class; later
 * BE_ALGO_AUTO calls of that class use it.  `out` receives the labels.  choice: 0..2 = tile
 * shape of the union-find form, 16 = iterative form. */
int be_autotune2d(be_ctx *ctx, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
                  int threshold, int32_t *out, int64_t out_pitch, int *choice, void *stream);
int be_autotune3d(be_ctx *ctx, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int threshold,
                  int32_t *out, int *choice, void *stream);
/* Tuning table to / from a text file ("class algo shape microseconds" per line). */
int be_tune_save(const be_ctx *ctx, const char *path);
int be_tune_load(be_ctx *ctx, const char *path);

/* ---- Batched labeling (no counterpart in the reference, which loops over files on the host,
 * main.cpp:309-340) ------------------------------------------------------------------------------
 * One batch = any mix of 2D images and 3D volumes of any sizes, labeled by ONE launch sequence
 * captured in a CUDA graph: persistent CTAs pull tiles of all images from atomic work queues.
 * Buffers stay owned by the caller and must stay valid while the batch exists (the graph holds
 * their addresses). */
typedef struct be_image {
    const uint8_t *in;   /* 2D: rows x cols, in_pitch bytes per row; 3D: dense [d0][d1][d2] */
    int32_t *out;        /* int32 labels, same layout (2D: out_pitch elements per row) */
    int64_t in_pitch;
    int64_t out_pitch;
    int32_t dims[3];     /* 2D: {rows, cols, 0}; 3D: {d0, d1, d2} */
    int32_t threshold;   /* foreground is pixel > threshold */
} be_image;

enum { BE_BATCH_ONE_CTA_PER_TILE = 0x100 /* no persistent CTAs / work queue */ };

typedef struct be_batch be_batch;
int be_batch_create(be_ctx *ctx, const be_image *imgs, int n, int flags, be_batch **batch);
/* Launches the batch's graph on `stream` (asynchronous). */
int be_batch_run(be_batch *batch, void *stream);
/* Component count of every image, in the caller's order (synchronizes `stream`). */
int be_batch_counts(be_batch *batch, int64_t *counts, void *stream);
/* Times the 2D tile shapes and persistent vs one-CTA-per-tile launches on this batch and keeps
 * the fastest graph; *choice = shape | flags. */
int be_batch_tune(be_batch *batch, void *stream, int *choice);
int be_batch_destroy(be_batch *batch);

/* ---- Serving loop (no counterpart in the reference) -----------------------------------------
 * Continuous batching: requests submitted from any thread are admitted while their device memory
 * fits the budget (default: 80% of free device memory at creation) and labeled in batches by the
 * persistent-kernel pipeline; requests arriving while batches run join the next one; `lanes`
 * batches can be in flight on separate streams.  Device buffers come from a memory pool that keeps
 * its memory.  Results are the same as labeling each image alone. */
enum { BE_REQ_DEVICE_BUFFERS = 1 /* in / out are device pointers: no copies */ };

typedef struct be_request {
    const uint8_t *in;   /* host (pinned for full overlap) or device, dense */
    int32_t *out;        /* same kind as `in`, dense int32 labels */
    int32_t dims[3];     /* 2D: {rows, cols, 0}; 3D: {d0, d1, d2} */
    int32_t threshold;
    int32_t flags;       /* BE_REQ_* */
} be_request;

typedef struct be_result {
    int32_t status;      /* BE_OK, BE_ERR_OOM, BE_ERR_BUSY (can never fit), BE_ERR_CANCELLED, ... */
    int64_t n_components;
    double latency_us;   /* submit -> completion */
} be_result;

typedef struct be_server_config {
    int32_t device;
    int64_t max_device_bytes;          /* 0: 80% of the free memory at creation */
    int32_t lanes;                     /* batches in flight at once (streams) */
    int32_t max_batch;                 /* requests per batch */
    int32_t inject_alloc_failure_every; /* tests: every n-th device allocation fails (0 = off) */
} be_server_config;

typedef struct be_serve_stats {
    int64_t completed, rejected, failed, batches, pixels;
    double p50_us, p99_us, mean_us, wall_s;
    int64_t device_bytes_in_use, device_bytes_budget;
} be_serve_stats;

typedef struct be_server be_server;
void be_server_default_config(be_server_config *cfg);
int be_server_create(const be_server_config *cfg, be_server **server);
int be_server_submit(be_server *server, const be_request *req, uint64_t *id);
/* Waits for request `id` (timeout_us < 0: no limit; BE_ERR_TIMEOUT when it runs out) and returns
 * its status; the request is forgotten afterwards. */
int be_server_wait(be_server *server, uint64_t id, int64_t timeout_us, be_result *result);
/* Queued requests are dropped; a running one completes on the GPU but is reported cancelled. */
int be_server_cancel(be_server *server, uint64_t id);
int be_server_stats(be_server *server, be_serve_stats *stats);
int be_server_reset_stats(be_server *server);
/* Drains every submitted request, then stops. */
int be_server_destroy(be_server *server);

/* 2D labeling that allocates no memory (no counterpart in the reference).  For callers that
 * cannot call cudaMalloc -- a framework that already owns the device memory pool, a latency-bound
 * loop that must not stall on cudaMalloc's implicit synchronization, a plugin host that forbids
 * allocation.  Same computation and result as be_label2d (8-connectivity, union-find form), but the
 * scratch is one fixed array inside the library's device image, held by every GPU that loads the
 * library until exit.  Limit: at most 1024 tiles of 64 x 256 pixels and rows x ceil(cols / 256) <=
 * 65536 (4096 x 4096 fits); larger images return BE_ERR_TOO_LARGE.  The first call on a device
 * looks the array's device address up (cudaGetSymbolAddress) with that device current; make it
 * before any stream capture.  All calls share the array: calls whose work overlaps on the GPU
 * race, so order them (one stream, or events).  n_components, if not NULL, receives K after a
 * synchronization of `stream`.  No context, so no be_last_error message: the status says it all. */
int be_label2d_noalloc(const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols, int threshold,
                       int32_t *out, int64_t out_pitch, int64_t *n_components, void *stream);

/* ---- Ingest and egress on the device (the steps either side of the labeling path) ---------------
 * be_to_gray replaces ILabeling::RGB2Gray (Labeling2015/src/LabelingTools.cpp:39-49): channels 1
 * (gray) or 3 (RGB order, cv::COLOR_RGB2GRAY), then with BE_GRAY_BINARIZE the reference's fixed
 * threshold, Y > 8 ? 255 : 0.  The gray weights are OpenCV 3.0.0's, the version the reference
 * builds against: Y = (4899 R + 9617 G + 1868 B + 2^13) >> 14; with BE_GRAY_OPENCV4 those of
 * OpenCV 4: Y = (9798 R + 19235 G + 3735 B + 2^14) >> 15 (within one gray level of the former).
 * flags = 0 / 1 keeps the meaning of the former `binarize` argument.  Pitches in bytes. */
#define BE_GRAY_BINARIZE 1
#define BE_GRAY_OPENCV4 2
int be_to_gray(be_ctx *ctx, const uint8_t *in, int64_t in_pitch, int channels, int32_t rows, int32_t cols,
               int flags, uint8_t *out, int64_t out_pitch, void *stream);

/* be_stack_slices replaces the slice stacking of Read3DImage (Labeling2015/main.cpp:172-212):
 * `planes` slices of rows x cols pixels (channels 1 or 3, packed slice after slice) become the
 * volume [rows][cols][planes] -- the slice index is the fastest dimension, as the reference
 * stacks them -- each voxel binarized as RGB2Gray does (0 / 255).  rows <= 65535. */
int be_stack_slices(be_ctx *ctx, const uint8_t *slices, int channels, int32_t rows, int32_t cols,
                    int32_t planes, uint8_t *volume, void *stream);

/* be_labels_to_rgb replaces LabelsToRGB (Labeling2015/main.cpp:248-286): 3 bytes per label, the
 * background black, every other label a colour hashed from (label, seed).  The reference draws
 * its colours with std::rand in label order, so its colours are not reproducible; this map is
 * deterministic and needs no table.  n labels in, 3 n bytes out. */
int be_labels_to_rgb(be_ctx *ctx, const int32_t *labels, int64_t n, uint32_t seed, uint8_t *rgb, void *stream);

/* be_volume_to_rgb_planes replaces the plane loop of Write3DLabels (Labeling2015/main.cpp:290-305):
 * the label volume [d0][d1][d2] becomes d2 colour planes of d0 x d1 RGB pixels, plane after plane,
 * coloured as be_labels_to_rgb.  d0 <= 65535. */
int be_volume_to_rgb_planes(be_ctx *ctx, const int32_t *labels, int32_t d0, int32_t d1, int32_t d2, uint32_t seed,
                            uint8_t *rgb, void *stream);

/* ---- Slab split of one image (no counterpart in the reference, which labels one image on one
 * device, LabelingAlgs.cpp:989-1084) ----------------------------------------------------------
 * A slab is a band of consecutive rows of a 2D image, or of consecutive planes along d0 of a
 * volume, labeled on its own by be_label2d / be_label3d (on its own GPU, or in turn on one GPU):
 * its labels are 1..counts[s] in first-pixel order within the slab.  One exchange step joins the
 * slabs: gather every slab's first and last row (plane) of labels and its count, call
 * be_slab_merge (host only, identical on every rank), then be_slab_relabel on each slab.
 *
 * be_slab_merge: n_slabs slabs in image order; a border row (plane) is plane_rows x plane_cols
 * labels (2D: plane_rows = 1, plane_cols = cols; 3D: d1 x d2).  tops / bottoms hold the slabs'
 * first / last rows, slab after slab.  Pieces touching across a border are joined
 * (8-connectivity across a row, 26-connectivity across a plane).  Out: offsets[s] (root pieces
 * of the slabs before s), *n_total (components of the whole image), and per slab the ascending
 * local labels of its pieces that were joined under an earlier piece, with their final labels:
 * joined_labels / joined_targets[joined_start[s] .. joined_start[s + 1]).  cap = capacity of the
 * joined arrays; 2 * plane_rows * plane_cols * n_slabs always suffices.  BE_ERR_INVALID on bad
 * sizes, labels outside 0..counts[s], a cap too small or more than INT32_MAX components. */
int be_slab_merge(int32_t n_slabs, int32_t plane_rows, int32_t plane_cols, const int64_t *counts,
                  const int32_t *tops, const int32_t *bottoms, int64_t *offsets, int64_t *n_total,
                  int32_t *joined_labels, int32_t *joined_targets, int64_t *joined_start, int64_t cap);

/* be_slab_relabel: maps the local labels of one slab (device array of n_rows rows of cols labels,
 * pitch in elements; a 3D slab of p planes is p * d1 rows of d2) to the whole image's labels:
 * joined labels to their targets, every other label l in 1..count to offset + l - (joined labels
 * below l).  joined_labels (ascending) / joined_targets are HOST arrays of n_joined entries, as
 * be_slab_merge returns them for this slab; pageable memory is read before the call returns,
 * pinned memory must stay valid until the stream reaches the call.  Values outside 0..count are
 * left unchanged.  The context's slab scratch is shared by its calls: order calls that overlap.
 * The scratch grows inside the call when count or n_joined exceed what the context holds (a
 * device allocation, which synchronizes the device); be_slab_reserve sizes it beforehand. */
int be_slab_relabel(be_ctx *ctx, int32_t *labels, int64_t n_rows, int32_t cols, int64_t pitch, int64_t count,
                    int64_t offset, const int32_t *joined_labels, const int32_t *joined_targets, int32_t n_joined,
                    void *stream);

/* be_slab_reserve: sizes the context's slab scratch for later be_slab_relabel calls of up to
 * max_count local labels and max_joined joined labels, so that those calls allocate nothing.
 * A slab of n pixels has at most n / 2 + 1 components (8-connectivity), and at most
 * 2 x (border row or plane size) joined labels. */
int be_slab_reserve(be_ctx *ctx, int64_t max_count, int64_t max_joined);

/* Report of the bounds-checked debug build (-DBE_BOUNDS_CHECK; no counterpart in the
 * reference): out3 = {site, value low, value high} of the first failed index check of the last
 * 2D (dims = 2) or 3D (dims = 3) union-find call, all zero when none failed.  Normal builds
 * perform no checks and always report zeros. */
int be_check_status(be_ctx *ctx, int dims, uint32_t *out3);

/* Per-launch timing of plain calls (no counterpart in the reference, whose stopwatch covers the
 * whole DoOCLLabel call, LabelingTools.cpp:118-125).  When enabled, be_label2d / be_label3d
 * record a CUDA event before and after each of their launches; be_stage_times then returns the
 * device time of each launch of the last call in ms (it waits for that call's last event). */
int be_set_stage_timing(be_ctx *ctx, int enable);
int be_stage_times(be_ctx *ctx, float *ms, int max_stages, int *n_stages);

#ifdef __cplusplus
}
#endif

#endif /* BE_B200_H_ */

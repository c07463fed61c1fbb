// be_tune.cu -- the autotuner: chooses, per image size class, between the union-find pipeline in
// each 2D tile shape and the iterative scan/analyze form, by timing them on the caller's input.
//
// Choices are kept per context in a small table keyed by size class (2D: the two side lengths
// rounded down to powers of two; 3D: the voxel count rounded down to a power of two) and can be
// saved to / loaded from a text file.  BE_ALGO_AUTO calls look the table up; without an entry they
// use the union-find form in the default shape.  Every candidate produces the same labels (the
// canonical result does not depend on the schedule), which the tuner checks.
#include "be.h"
#include "be_api_internal.h"
#include "be_kernels.h"

#include <cstdio>
#include <vector>

namespace be {

namespace {

int floor_log2(int64_t v)
{
    int s = 0;
    while ((int64_t(2) << s) <= v) ++s;
    return s;
}

uint32_t class2d(int rows, int cols) { return (2u << 16) | (uint32_t(floor_log2(rows)) << 8) | uint32_t(floor_log2(cols)); }
uint32_t class3d(int64_t n) { return (3u << 16) | uint32_t(floor_log2(n)); }

const TuneEntry *lookup(const be_ctx *c, uint32_t cls)
{
    for (const TuneEntry &e : c->tune)
        if (e.cls == cls) return &e;
    return nullptr;
}

void store(be_ctx *c, uint32_t cls, int algo, int shape, float us)
{
    for (TuneEntry &e : c->tune)
        if (e.cls == cls) {
            e.algo = algo;
            e.shape = shape;
            e.us = us;
            return;
        }
    c->tune.push_back(TuneEntry{cls, algo, shape, us});
}

}  // namespace

void pick2d(const be_ctx *c, int rows, int cols, int algo_in, int *algo, int *shape)
{
    const TuneEntry *e = lookup(c, class2d(rows, cols));
    *shape = e && e->algo == BE_ALGO_UF ? e->shape : 0;
    if (algo_in != BE_ALGO_AUTO) *algo = algo_in;
    else *algo = e ? e->algo : BE_ALGO_UF;
}

void pick3d(const be_ctx *c, int64_t n, int algo_in, int *algo)
{
    const TuneEntry *e = lookup(c, class3d(n));
    if (algo_in != BE_ALGO_AUTO) *algo = algo_in;
    else *algo = e ? e->algo : BE_ALGO_UF;
}

}  // namespace be

using namespace be;

extern "C" {

int be_autotune2d(be_ctx *c, const uint8_t *in, int64_t in_pitch, int32_t rows, int32_t cols,
                  int threshold, int32_t *out, int64_t out_pitch, int *choice, void *stream)
{
    if (!c || !in || !out || rows <= 0 || cols <= 0) return BE_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
        return set_error(c, BE_ERR_CUDA, "be_autotune2d: event creation failed");
    struct Cand { int algo, shape; };
    std::vector<Cand> cands;
    for (int sh = 0; sh < kNumShapes2D; ++sh) cands.push_back({BE_ALGO_UF, sh});
    cands.push_back({BE_ALGO_ITER, 0});
    const uint32_t cls = class2d(rows, cols);
    float best = 1e30f;
    int best_i = 0, rc = BE_OK;
    int64_t k0 = -1;
    std::vector<int32_t> ref, cur;
    const size_t n = size_t(rows) * cols;
    for (size_t i = 0; i < cands.size() && rc == BE_OK; ++i) {
        store(c, cls, cands[i].algo, cands[i].shape, 0.f);   // route AUTO to this candidate
        float ms = 0;
        int64_t k = 0;
        for (int rep = 0; rep < 3 && rc == BE_OK; ++rep) {   // 1 warm-up + 2 timed
            cudaEventRecord(a, s);
            rc = be_label2d(c, in, in_pitch, rows, cols, threshold, BE_COH_DEFAULT, BE_ALGO_AUTO, out,
                            out_pitch, &k, stream);
            cudaEventRecord(b, s);
            cudaEventSynchronize(b);
            float t = 0;
            cudaEventElapsedTime(&t, a, b);
            if (rep) ms += t;
        }
        if (rc == BE_ERR_INVALID && cands[i].algo == BE_ALGO_ITER) {   // outside its key space
            c->err.clear();
            rc = BE_OK;
            continue;
        }
        if (rc) break;
        // Every candidate must reproduce the first one's labels (schedule independence).
        cur.resize(n);
        cudaMemcpy2D(cur.data(), cols * sizeof(int32_t), out, out_pitch * sizeof(int32_t),
                     cols * sizeof(int32_t), rows, cudaMemcpyDeviceToHost);
        if (i == 0) {
            ref.swap(cur);
            k0 = k;
        } else if (k != k0 || cur != ref) {
            rc = set_error(c, BE_ERR_CUDA, "be_autotune2d: candidate %d/%d disagrees", cands[i].algo,
                           cands[i].shape);
            break;
        }
        if (ms < best) {
            best = ms;
            best_i = int(i);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    store(c, cls, cands[best_i].algo, cands[best_i].shape, best * 500.f);
    if (choice) *choice = cands[best_i].algo == BE_ALGO_ITER ? 16 : cands[best_i].shape;
    return BE_OK;
}

int be_autotune3d(be_ctx *c, const uint8_t *in, int32_t d0, int32_t d1, int32_t d2, int threshold,
                  int32_t *out, int *choice, void *stream)
{
    if (!c || !in || !out || d0 <= 0 || d1 <= 0 || d2 <= 0) return BE_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
        return set_error(c, BE_ERR_CUDA, "be_autotune3d: event creation failed");
    const uint32_t cls = class3d(int64_t(d0) * d1 * d2);
    const int algos[2] = {BE_ALGO_UF, BE_ALGO_ITER};
    float best = 1e30f;
    int best_algo = BE_ALGO_UF, rc = BE_OK;
    for (int i = 0; i < 2 && rc == BE_OK; ++i) {
        float ms = 0;
        for (int rep = 0; rep < 3 && rc == BE_OK; ++rep) {
            cudaEventRecord(a, s);
            rc = be_label3d(c, in, d0, d1, d2, threshold, algos[i], out, nullptr, stream);
            cudaEventRecord(b, s);
            cudaEventSynchronize(b);
            float t = 0;
            cudaEventElapsedTime(&t, a, b);
            if (rep) ms += t;
        }
        if (rc == BE_ERR_INVALID && algos[i] == BE_ALGO_ITER) {
            c->err.clear();
            rc = BE_OK;
            continue;
        }
        if (rc == BE_OK && ms < best) {
            best = ms;
            best_algo = algos[i];
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    store(c, cls, best_algo, 0, best * 500.f);
    if (choice) *choice = best_algo == BE_ALGO_ITER ? 16 : 0;
    return BE_OK;
}

int be_tune_save(const be_ctx *c, const char *path)
{
    if (!c || !path) return BE_ERR_INVALID;
    FILE *f = std::fopen(path, "w");
    if (!f) return BE_ERR_INVALID;
    std::fprintf(f, "# be_b200 tuning table: class algo shape us\n");
    for (const TuneEntry &e : c->tune) std::fprintf(f, "%u %d %d %.3f\n", e.cls, e.algo, e.shape, e.us);
    std::fclose(f);
    return BE_OK;
}

int be_tune_load(be_ctx *c, const char *path)
{
    if (!c || !path) return BE_ERR_INVALID;
    FILE *f = std::fopen(path, "r");
    if (!f) return BE_ERR_INVALID;
    char line[256];
    int rc = BE_OK;
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#') continue;
        unsigned cls;
        int algo, shape;
        float us;
        if (std::sscanf(line, "%u %d %d %f", &cls, &algo, &shape, &us) != 4 || algo < BE_ALGO_UF ||
            algo > BE_ALGO_ITER || shape < 0 || shape >= kNumShapes2D) {
            rc = BE_ERR_INVALID;
            break;
        }
        store(c, cls, algo, shape, us);
    }
    std::fclose(f);
    return rc;
}

}  // extern "C"

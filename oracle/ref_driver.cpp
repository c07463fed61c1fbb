// ref_driver.cpp -- host drivers that run the reference's own OpenCL kernels
// (Labeling2015/src/LabelingAlgs.cl, compiled unmodified as C++ through ref_shim/cl_as_cpp.hpp)
// with the reference's host flow, serially on the CPU.  Built by oracle/Makefile into
// oracle/_ref/libref_be.so.  TEST INFRASTRUCTURE ONLY: used to pin the oracle restatement
// (oracle/be_oracle.c) and to generate the golden fixtures under tests/golden/.
//
// Each driver reproduces, in order: the host padding of IOCLLabeling(3D)::Label
// (Labeling2015/src/LabelingTools.cpp:98-132, 160-221), the buffer set-up and kernel sequence of the
// algorithm class (Labeling2015/src/LabelingAlgs.cpp), and the crop back to the input size.  Buffers
// that the reference creates without initialisation are zero-filled (the values the kernels need).
#include "cl_as_cpp.hpp"

namespace refcl {
thread_local size_t gid[3];
thread_local size_t gsz[3];
int nthreads = 1;
}  // namespace refcl

#include REF_CL

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

std::vector<uchar> pad2d(const uint8_t *img, long rows, long cols, long pitch, int thr, long W,
                         long H)
{
    std::vector<uchar> p((size_t)W * H, 0);
    for (long y = 0; y < rows; ++y)
        for (long x = 0; x < cols; ++x) p[(size_t)y * W + x] = img[y * pitch + x] > thr ? 255 : 0;
    return p;
}

}  // namespace

extern "C" {

// TOCLLabelEquivalenceX2::DoOCLLabel (LabelingAlgs.cpp:1067-1084) on the IOCLLabeling::Label
// padded image; writes the reference's label values cropped to rows x cols.
int ref_lbeq2_raw(const uint8_t *img, long rows, long cols, long pitch, int thr, uint32_t *out)
{
    if (rows <= 0 || cols <= 0) return -1;
    const long W = (cols >> 5 << 5) + 32, H = (rows >> 5 << 5) + 32;
    std::vector<uchar> pix = pad2d(img, rows, cols, pitch, thr, W, H);
    std::vector<TLabel> labels((size_t)W * H, 0);
    // InitSPixels (LabelingAlgs.cpp:989-1010)
    const size_t spW = (size_t)std::ceil((float)W / 2), spH = (size_t)std::ceil((float)H / 2);
    std::vector<TLabel> sLabels(spW * spH, 0);
    std::vector<char> sConn(spW * spH, 0);
    const size_t initSz[2] = {spW, spH};
    ref_ndrange(2, initSz, [&] {
        LBEQ2_Init(pix.data(), sLabels.data(), sConn.data(), (uint)W, (uint)H);
    });
    // LabelSPixels (LabelingAlgs.cpp:1014-1039)
    const size_t anSz[1] = {spW * spH};
    for (;;) {
        char noChanges = 1;
        ref_ndrange(2, initSz, [&] { LBEQ2_Scan(sLabels.data(), sConn.data(), &noChanges); });
        if (noChanges) break;
        ref_ndrange(1, anSz, [&] { LBEQ2_Analyze(sLabels.data()); });
    }
    // SetFinalLabels (LabelingAlgs.cpp:1043-1055)
    const size_t finSz[2] = {(size_t)W, (size_t)H};
    ref_ndrange(2, finSz, [&] { LBEQ2_SetFinalLabels(pix.data(), labels.data(), sLabels.data()); });
    for (long y = 0; y < rows; ++y)
        std::memcpy(out + y * cols, labels.data() + (size_t)y * W, sizeof(uint32_t) * cols);
    return 0;
}

// TOCLBlockEquivalence3D::DoOCLLabel3D (LabelingAlgs.cpp:1520-1536) on the CopyAlignImg volume
// (LabelingTools.cpp:160-176); the output is cropped back to d0 x d1 x d2 (the reference itself
// returns the padded volume, LabelingTools.cpp:217-220).
// With usec, the time of the kernel sequence alone is written there (the span the reference's
// stopwatch covers, LabelingTools.cpp:206-214).
int ref_bleq3d_timed(const uint8_t *vol, long d0, long d1, long d2, int thr, uint32_t *out, double *usec)
{
    if (d0 <= 0 || d1 <= 0 || d2 <= 0) return -1;
    const long X = ((d0 + 4) >> 5 << 5) + 32, Y = ((d1 + 4) >> 5 << 5) + 32,
               Z = ((d2 + 4) >> 5 << 5) + 32;
    std::vector<uchar> pix((size_t)X * Y * Z, 0);
    for (long x = 0; x < d0; ++x)
        for (long y = 0; y < d1; ++y)
            for (long z = 0; z < d2; ++z)
                pix[((size_t)(x + 2) * Y + (y + 2)) * Z + (z + 2)] =
                    vol[(x * d1 + y) * d2 + z] > thr ? 255 : 0;
    std::vector<TLabel> labels(pix.size(), 0);
    const size_t sp[3] = {(size_t)X >> 1, (size_t)Y >> 1, (size_t)Z >> 1};
    std::vector<TLabel> sLabels(sp[0] * sp[1] * sp[2], 0);
    std::vector<int> sConn(sLabels.size(), 0);
    const auto t0 = std::chrono::steady_clock::now();
    ref_ndrange(3, sp, [&] { BLEQ3D_Init(pix.data(), sLabels.data(), sConn.data()); });
    const size_t anSz[1] = {sLabels.size()};
    for (;;) {
        char noChanges = 1;
        ref_ndrange(3, sp, [&] { BLEQ3D_Scan(sLabels.data(), sConn.data(), &noChanges); });
        if (noChanges) break;
        ref_ndrange(1, anSz, [&] { BLEQ3D_Analyze(sLabels.data()); });
    }
    const size_t fin[3] = {(size_t)X, (size_t)Y, (size_t)Z};
    ref_ndrange(3, fin, [&] { BLEQ3D_SetFinalLabels(pix.data(), labels.data(), sLabels.data()); });
    if (usec)
        *usec = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    for (long x = 0; x < d0; ++x)
        for (long y = 0; y < d1; ++y)
            for (long z = 0; z < d2; ++z)
                out[(x * d1 + y) * d2 + z] = labels[((size_t)(x + 2) * Y + (y + 2)) * Z + (z + 2)];
    return 0;
}

int ref_bleq3d_raw(const uint8_t *vol, long d0, long d1, long d2, int thr, uint32_t *out)
{
    return ref_bleq3d_timed(vol, d0, d1, d2, thr, out, nullptr);
}

// Work-item threads of every driver here: 1 = serial (the default), 0 = all OpenMP threads.
int ref_set_threads(int n)
{
    refcl::nthreads = n > 0 ? n : omp_get_max_threads();
    return refcl::nthreads;
}

// TOCLLabelDistribution::DoOCLLabel (LabelingAlgs.cpp:867-942): DistrInitKernel, then
// DistrScanKernel / DistrAnalizeKernel until no change.  coh: 0 = COH_4, 1 = COH_8,
// 2 = COH_DEFAULT (the CLI default, which the kernel treats as 4-connectivity).
int ref_distr2d_raw(const uint8_t *img, long rows, long cols, long pitch, int thr, int coh,
                    uint32_t *out)
{
    if (rows <= 0 || cols <= 0) return -1;
    const long W = (cols >> 5 << 5) + 32, H = (rows >> 5 << 5) + 32;
    std::vector<uchar> pix = pad2d(img, rows, cols, pitch, thr, W, H);
    std::vector<TLabel> labels((size_t)W * H, 0);
    const size_t n[1] = {(size_t)W * H};
    ref_ndrange(1, n, [&] { DistrInitKernel(pix.data(), labels.data()); });
    for (;;) {
        char noChanges = 1;
        ref_ndrange(1, n, [&] {
            DistrScanKernel(labels.data(), (uint)W, (uint)H, (TCoherence)coh, &noChanges);
        });
        if (noChanges) break;
        ref_ndrange(1, n, [&] { DistrAnalizeKernel(labels.data()); });
    }
    for (long y = 0; y < rows; ++y)
        std::memcpy(out + y * cols, labels.data() + (size_t)y * W, sizeof(uint32_t) * cols);
    return 0;
}

// TOCLRunEquivLabeling::DoOCLLabel (LabelingAlgs.cpp:1226-1268): REInitRuns, REFindRuns,
// REFindNeib, then REScan / REAnalize until no change, RELabel -- one work-item per row of the
// IOCLLabeling::Label padded image; the labels are cropped to rows x cols.
int ref_runeq2d_raw(const uint8_t *img, long rows, long cols, long pitch, int thr, uint32_t *out)
{
    if (rows <= 0 || cols <= 0) return -1;
    const long W = (cols >> 5 << 5) + 32, H = (rows >> 5 << 5) + 32;
    std::vector<uchar> pix = pad2d(img, rows, cols, pitch, thr, W, H);
    std::vector<TLabel> labels((size_t)W * H, 0);
    std::vector<TRun> runs((size_t)H * (W >> 1));
    std::memset(runs.data(), 0, runs.size() * sizeof(TRun));
    std::vector<uint> runNum((size_t)H, 0);
    const size_t n[1] = {(size_t)H};
    ref_ndrange(1, n, [&] { REInitRunsKernel(runNum.data()); });
    ref_ndrange(1, n, [&] { REFindRunsKernel(pix.data(), runs.data(), runNum.data(), (uint)W); });
    ref_ndrange(1, n, [&] { REFindNeibKernel(runs.data(), runNum.data(), (uint)W); });
    for (;;) {
        char noChanges = 1;
        ref_ndrange(1, n, [&] { REScanKernel(runs.data(), runNum.data(), (uint)W, &noChanges); });
        if (noChanges) break;
        ref_ndrange(1, n, [&] { REAnalizeKernel(runs.data(), runNum.data(), (uint)W); });
    }
    ref_ndrange(1, n, [&] { RELabelKernel(runs.data(), runNum.data(), labels.data(), (uint)W); });
    for (long y = 0; y < rows; ++y)
        std::memcpy(out + y * cols, labels.data() + (size_t)y * W, sizeof(uint32_t) * cols);
    return 0;
}

// TOCLLabelEquivalence3D::DoOCLLabel3D (LabelingAlgs.cpp:1362-1396) on the CopyAlignImg volume.
int ref_lbeq3d_raw(const uint8_t *vol, long d0, long d1, long d2, int thr, uint32_t *out)
{
    if (d0 <= 0 || d1 <= 0 || d2 <= 0) return -1;
    const long X = ((d0 + 4) >> 5 << 5) + 32, Y = ((d1 + 4) >> 5 << 5) + 32,
               Z = ((d2 + 4) >> 5 << 5) + 32;
    std::vector<uchar> pix((size_t)X * Y * Z, 0);
    for (long x = 0; x < d0; ++x)
        for (long y = 0; y < d1; ++y)
            for (long z = 0; z < d2; ++z)
                pix[((size_t)(x + 2) * Y + (y + 2)) * Z + (z + 2)] =
                    vol[(x * d1 + y) * d2 + z] > thr ? 255 : 0;
    std::vector<TLabel> labels(pix.size(), 0);
    const size_t n[1] = {pix.size()};
    const size_t sz[3] = {(size_t)X, (size_t)Y, (size_t)Z};
    ref_ndrange(1, n, [&] { LBEQ3D_InitKernel(pix.data(), labels.data()); });
    for (;;) {
        char noChanges = 1;
        ref_ndrange(3, sz, [&] { LBEQ3D_ScanKernel(labels.data(), &noChanges); });
        if (noChanges) break;
        ref_ndrange(1, n, [&] { LBEQ3D_AnalyzeKernel(labels.data()); });
    }
    for (long x = 0; x < d0; ++x)
        for (long y = 0; y < d1; ++y)
            for (long z = 0; z < d2; ++z)
                out[(x * d1 + y) * d2 + z] = labels[((size_t)(x + 2) * Y + (y + 2)) * Z + (z + 2)];
    return 0;
}

}  // extern "C"

// ref_cpu.cpp -- C-ABI driver for the reference's own OpenMP CPU labelers, compiled from the
// reference sources where they lie (Labeling2015/src/LabelingAlgs.cpp, LabelingTools.cpp,
// stopwatch_win.cpp, cvlabeling_imagelab.cpp) against the stand-in headers under ref_shim/.
// TEST INFRASTRUCTURE ONLY: it is the CPU baseline the benchmark times beside the GPU path and a
// second opinion for the parity tests; nothing in the product links it.
//
// The CPU slots of the reference's algorithm registry (Labeling2015/main.cpp:100-131):
//   "bleq"  TLabelEquivalenceX2  (block equivalence, 2x2 blocks, 8-connectivity)
//   "lbeq"  TLabelDistribution   (pixel label equivalence, 4 or 8 connectivity)
//   "runeq" TRunEqivLabeling     (run equivalence, 8-connectivity)
//   "gr-block" TBlockGranaLabeling
// Each is run through ILabeling::Label (LabelingTools.cpp:19-36): binarize at the fixed
// threshold 8, label, return the reference's own stopwatch time.
#include "LabelingAlgs.hpp"

#include <opencv2/imgproc/imgproc.hpp>

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>

// OpenCL entry points: the reference's OpenCL classes are compiled but never constructed here.
extern "C" {
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void *, cl_int *e)
{
    if (e) *e = CL_INVALID_OPERATION;
    return nullptr;
}
cl_int clReleaseMemObject(cl_mem) { return CL_INVALID_OPERATION; }
cl_kernel clCreateKernel(cl_program, const char *, cl_int *e)
{
    if (e) *e = CL_INVALID_OPERATION;
    return nullptr;
}
cl_int clReleaseKernel(cl_kernel) { return CL_INVALID_OPERATION; }
cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void *) { return CL_INVALID_OPERATION; }
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t *, const size_t *,
                              const size_t *, cl_uint, const cl_event *, cl_event *)
{
    return CL_INVALID_OPERATION;
}
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void *, cl_uint,
                           const cl_event *, cl_event *)
{
    return CL_INVALID_OPERATION;
}
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void *, cl_uint,
                            const cl_event *, cl_event *)
{
    return CL_INVALID_OPERATION;
}
cl_int clFinish(cl_command_queue) { return CL_INVALID_OPERATION; }
int InitOpenCL(clState *, clInitParams *) { return CL_INVALID_OPERATION; }
int TerminateOpenCL(clState *) { return CL_SUCCESS; }
int clInitKernel(cl_kernel *, const clState *, const char *) { return CL_INVALID_OPERATION; }
int clExecuteKernel(const clState *, const cl_kernel *, const void **, const size_t *, int, size_t, size_t, int)
{
    return CL_INVALID_OPERATION;
}
}  // extern "C"

// The three imgproc calls the sources name.  Only threshold() is on the labeling path.
namespace cv {
void cvtColor(const Mat &src, Mat &dst, int)
{
    Mat out(src.rows, src.cols, CV_8UC1);
    const int cn = src.channels();
    for (int r = 0; r < src.rows; ++r)
        for (int c = 0; c < src.cols; ++c) {
            const uchar *p = src.data + r * src.step[0] + c * src.step[1];
            // RGB order, ITU-R BT.601 weights of COLOR_RGB2GRAY, rounded to nearest.
            out.at<uchar>(r, c) = cn >= 3 ? uchar(0.299 * p[0] + 0.587 * p[1] + 0.114 * p[2] + 0.5) : p[0];
        }
    dst = out;
}

double threshold(const Mat &src, Mat &dst, double thresh, double maxval, int)
{
    Mat out;
    if (src.dims == 2) out = Mat(src.rows, src.cols, CV_8UC1);
    else out = Mat(src.dims, src.size, CV_8UC1);
    const size_t n = src.total();
    if (src.dims == 2) {
        for (int r = 0; r < src.rows; ++r)
            for (int c = 0; c < src.cols; ++c)
                out.at<uchar>(r, c) = src.at<uchar>(r, c) > thresh ? uchar(maxval) : 0;
    } else {
        for (size_t i = 0; i < n; ++i) out.data[i] = src.data[i] > thresh ? uchar(maxval) : 0;
    }
    dst = out;
    return thresh;
}

int connectedComponents(const Mat &, Mat &, int, int) { return -1; }
}  // namespace cv

namespace {

std::shared_ptr<LabelingTools::ILabeling> make_alg(const std::string &name)
{
    using namespace LabelingTools;
    if (name == "bleq") return std::make_shared<TLabelEquivalenceX2>();
    if (name == "lbeq") return std::make_shared<TLabelDistribution>();
    if (name == "runeq") return std::make_shared<TRunEqivLabeling>();
    if (name == "gr-block") return std::make_shared<TBlockGranaLabeling>();
    return nullptr;
}

}  // namespace

extern "C" {

// Labels a rows x cols gray image (row pitch `cols`) with the reference CPU algorithm `alg`:
// foreground is pixel > thr (the image is binarized to 0 / 255 before the call, so the
// reference's own fixed threshold at 8 keeps it), `threads` OpenMP threads (0 = all), coh 0 =
// COH_4, 1 = COH_8, 2 = COH_DEFAULT.  Writes the reference's raw int32 labels to out (rows x
// cols) and the reference's own stopwatch time of DoLabel in microseconds to *usec.  Returns 0,
// -1 for an unknown algorithm, -2 when the reference threw.
int ref_cpu_label2d(const char *alg, const uint8_t *img, int rows, int cols, int thr, int threads,
                    int coh, int32_t *out, double *usec)
{
    auto a = make_alg(alg ? alg : "");
    if (!a) return -1;
    try {
        cv::Mat pixels(rows, cols, CV_8UC1);
        const size_t n = size_t(rows) * cols;
        for (size_t i = 0; i < n; ++i) pixels.data[i] = img[i] > thr ? 255 : 0;
        cv::Mat labels;
        const LabelingTools::TTime t =
            a->Label(pixels, labels, char(threads), LabelingTools::TCoherence(coh));
        for (int r = 0; r < rows; ++r) std::memcpy(out + size_t(r) * cols, &labels.at<int32_t>(r, 0), size_t(cols) * 4);
        if (usec) *usec = double(t);
    } catch (...) {
        return -2;
    }
    return 0;
}

int ref_cpu_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

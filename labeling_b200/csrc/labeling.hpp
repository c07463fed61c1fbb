// labeling.hpp -- C++ host interface of the B200 labeler, shaped like the reference's labeler
// interface (Labeling2015/src/LabelingTools.hpp:35-73) so that code written against
// `ILabeling::Label(pixels, labels, threads, coh) -> TTime` drops in.  It sits on the C ABI of
// include/be.h; the reference's cv::Mat is replaced by the small TImage below (no OpenCV).
#pragma once

#include "be.h"

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace LabelingB200 {

typedef uint8_t TPixel;     // LabelingTools.hpp:38
typedef int32_t TLabel;     // labels are written as int32 (CV_32SC1 in the reference)
typedef uint32_t TTime;     // microseconds, LabelingTools.hpp:41

enum TCoherence { COH_4, COH_8, COH_DEFAULT };   // LabelingTools.hpp:45-50

const char MAX_THREADS = 0;

// A dense 2D (depth == 0) or 3D image; dims are {rows, cols} or {d0, d1, d2} with the last fastest,
// the layout of the reference's cv::Mat (main.cpp:191-203).
template <class T>
struct TImageT {
    int dims = 2;
    int size[3] = {0, 0, 0};
    int channels = 1;                 // 1 (gray) or 3 (RGB, 2D only)
    std::vector<T> data;
    bool empty() const { return data.empty(); }
    size_t total() const { return size_t(size[0]) * size[1] * (dims == 3 ? size[2] : 1); }
    int rows() const { return size[0]; }
    int cols() const { return size[1]; }
};
typedef TImageT<TPixel> TImage;
typedef TImageT<TLabel> TLabelImage;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// ILabeling (LabelingTools.hpp:58-73): Label() binarizes, labels and returns the labeling time in
// microseconds; errors are exceptions.
class ILabeling {
public:
    virtual ~ILabeling() = default;
    virtual TTime Label(const TImage &pixels, TLabelImage &labels, char threads = MAX_THREADS,
                        TCoherence coh = COH_DEFAULT) = 0;
    // RGB -> gray (cv::COLOR_RGB2GRAY weights) and the fixed threshold at 8 of the reference's
    // RGB2Gray (LabelingTools.cpp:39-49), as 0 / 255.
    static TImage RGB2Gray(const TImage &img);
};

// GPU block equivalence, 2D (the `bleq` GPU slot; replaces TOCLLabelEquivalenceX2).
class TCudaBlockEquivalence final : public ILabeling {
public:
    explicit TCudaBlockEquivalence(bool runOnGPU = true, int algo = BE_ALGO_AUTO, int device = 0);
    ~TCudaBlockEquivalence() override;
    TTime Label(const TImage &pixels, TLabelImage &labels, char threads = MAX_THREADS,
                TCoherence coh = COH_DEFAULT) override;
    TCudaBlockEquivalence(const TCudaBlockEquivalence &) = delete;
    TCudaBlockEquivalence &operator=(const TCudaBlockEquivalence &) = delete;
    be_ctx *context() const { return ctx_; }

private:
    be_ctx *ctx_ = nullptr;
    int algo_;
};

// GPU block equivalence, 3D (the `bleq -3` GPU slot; replaces TOCLBlockEquivalence3D).
class TCudaBlockEquivalence3D final : public ILabeling {
public:
    explicit TCudaBlockEquivalence3D(bool runOnGPU = true, int algo = BE_ALGO_AUTO, int device = 0);
    ~TCudaBlockEquivalence3D() override;
    TTime Label(const TImage &pixels, TLabelImage &labels, char threads = MAX_THREADS,
                TCoherence coh = COH_DEFAULT) override;
    TCudaBlockEquivalence3D(const TCudaBlockEquivalence3D &) = delete;
    TCudaBlockEquivalence3D &operator=(const TCudaBlockEquivalence3D &) = delete;

private:
    be_ctx *ctx_ = nullptr;
    int algo_;
};

// GPU run equivalence, 2D (the `runeq` GPU slot; replaces TOCLRunEquivLabeling,
// LabelingAlgs.cpp:1090-1268).  The reference's run kernels join runs that overlap in a column,
// which is 4-connectivity, whatever coherence is asked for, and it rejects COH_4 itself; this
// slot keeps both: COH_4 throws, anything else labels 4-connected, with the run-equivalence form
// (BE_ALGO_RUNS).
class TCudaRunEquivalence final : public ILabeling {
public:
    explicit TCudaRunEquivalence(bool runOnGPU = true, int device = 0);
    TTime Label(const TImage &pixels, TLabelImage &labels, char threads = MAX_THREADS,
                TCoherence coh = COH_DEFAULT) override;

private:
    TCudaBlockEquivalence inner_;
};

// The algorithm registry of the reference's demo (main.cpp:88-131) for the slots this library
// fills.  CPU slots stay empty: there is no CPU fallback.
struct Algs {
    std::string descr;
    std::function<std::shared_ptr<ILabeling>()> cpu;
    std::function<std::shared_ptr<ILabeling>(bool)> gpu;
    std::function<std::shared_ptr<ILabeling>()> cpu3d;
    std::function<std::shared_ptr<ILabeling>(bool)> gpu3d;
};
const std::map<std::string, Algs> &AlgList();

// SetLabelingAlg (main.cpp:373-395); throws when the algorithm or mode is not available.
std::shared_ptr<ILabeling> SetLabelingAlg(const std::string &name, bool useGPU, bool label3D);

}  // namespace LabelingB200

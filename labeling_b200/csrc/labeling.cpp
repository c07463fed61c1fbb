// labeling.cpp -- the C++ labeler interface over the C ABI (see labeling.hpp).
#include "labeling.hpp"

#include <cmath>

namespace LabelingB200 {

namespace {

void check(be_ctx *ctx, int rc, const char *where)
{
    if (rc != BE_OK) {
        std::string msg = std::string(where) + " : ";
        msg += ctx ? be_last_error(ctx) : "error";
        throw Error(rc, msg);
    }
}

}  // namespace

TImage ILabeling::RGB2Gray(const TImage &img)
{
    TImage out;
    out.dims = img.dims;
    for (int i = 0; i < 3; ++i) out.size[i] = img.size[i];
    out.channels = 1;
    const size_t n = img.total();
    out.data.resize(n);
    for (size_t i = 0; i < n; ++i) {
        int v;
        if (img.channels == 3) {
            const TPixel *p = &img.data[3 * i];
            v = int(std::lround(0.299 * p[0] + 0.587 * p[1] + 0.114 * p[2]));
        } else {
            v = img.data[i];
        }
        out.data[i] = v > 8 ? 255 : 0;   // cv::threshold(.., 8, 255, THRESH_BINARY)
    }
    return out;
}

TCudaBlockEquivalence::TCudaBlockEquivalence(bool runOnGPU, int algo, int device) : algo_(algo)
{
    if (!runOnGPU) throw Error(BE_ERR_INVALID, "TCudaBlockEquivalence : there is no CPU mode");
    check(nullptr, be_create(&ctx_, device), "TCudaBlockEquivalence : be_create");
}

TCudaBlockEquivalence::~TCudaBlockEquivalence() { be_destroy(ctx_); }

// IOCLLabeling::Label (LabelingTools.cpp:98-132) without the padding: binarize, label, time.
TTime TCudaBlockEquivalence::Label(const TImage &pixels, TLabelImage &labels, char, TCoherence coh)
{
    if (pixels.empty()) throw Error(BE_ERR_INVALID, "TCudaBlockEquivalence::Label : Input image is empty");
    if (pixels.dims != 2) throw Error(BE_ERR_INVALID, "TCudaBlockEquivalence::Label : Input image is not 2D");
    const TImage bin = RGB2Gray(pixels);
    labels.dims = 2;
    labels.size[0] = bin.size[0];
    labels.size[1] = bin.size[1];
    labels.size[2] = 0;
    labels.data.assign(bin.total(), 0);
    double us = 0;
    check(ctx_, be_label2d_host(ctx_, bin.data.data(), bin.cols(), bin.rows(), bin.cols(), 0, int(coh), algo_,
                                labels.data.data(), labels.cols(), nullptr, &us),
          "TCudaBlockEquivalence::Label");
    return TTime(us);
}

TCudaBlockEquivalence3D::TCudaBlockEquivalence3D(bool runOnGPU, int algo, int device) : algo_(algo)
{
    if (!runOnGPU) throw Error(BE_ERR_INVALID, "TCudaBlockEquivalence3D : there is no CPU mode");
    check(nullptr, be_create(&ctx_, device), "TCudaBlockEquivalence3D : be_create");
}

TCudaBlockEquivalence3D::~TCudaBlockEquivalence3D() { be_destroy(ctx_); }

// IOCLLabeling3D::Label (LabelingTools.cpp:180-221): 3-D input, default connectivity only; the
// volume is used as given (Read3DImage binarized its slices).
TTime TCudaBlockEquivalence3D::Label(const TImage &pixels, TLabelImage &labels, char, TCoherence coh)
{
    if (pixels.empty()) throw Error(BE_ERR_INVALID, "TCudaBlockEquivalence3D::Label : Input image is empty");
    if (pixels.dims != 3) throw Error(BE_ERR_INVALID, "TCudaBlockEquivalence3D::Label : Input image is not a 3D image");
    if (coh != COH_DEFAULT)
        throw Error(BE_ERR_INVALID,
                    "TCudaBlockEquivalence3D::Label : Only default coherence is supported for 3D labeling");
    labels.dims = 3;
    for (int i = 0; i < 3; ++i) labels.size[i] = pixels.size[i];
    labels.data.assign(pixels.total(), 0);
    double us = 0;
    check(ctx_, be_label3d_host(ctx_, pixels.data.data(), pixels.size[0], pixels.size[1], pixels.size[2], 0, algo_,
                                labels.data.data(), nullptr, &us),
          "TCudaBlockEquivalence3D::Label");
    return TTime(us);
}

TCudaRunEquivalence::TCudaRunEquivalence(bool runOnGPU, int device) : inner_(runOnGPU, BE_ALGO_RUNS, device) {}

TTime TCudaRunEquivalence::Label(const TImage &pixels, TLabelImage &labels, char threads, TCoherence coh)
{
    if (coh == COH_4)   // as TOCLRunEquivLabeling::DoOCLLabel (LabelingAlgs.cpp:1229)
        throw Error(BE_ERR_INVALID, "TCudaRunEquivalence::Label : 4x connectivity is not implemented for this method");
    return inner_.Label(pixels, labels, threads, COH_4);
}

const std::map<std::string, Algs> &AlgList()
{
    static const std::map<std::string, Algs> list = {
        {"bleq",
         {"Block equivalence by Zavalishin et.al. 2016 (B200)", nullptr,
          [](bool gpu) { return std::make_shared<TCudaBlockEquivalence>(gpu, BE_ALGO_AUTO); }, nullptr,
          [](bool gpu) { return std::make_shared<TCudaBlockEquivalence3D>(gpu, BE_ALGO_AUTO); }}},
        {"lbeq",
         {"Label equivalence by Kalentev et.al. 2012 (pixel level, B200)", nullptr,
          [](bool gpu) { return std::make_shared<TCudaBlockEquivalence>(gpu, BE_ALGO_PIXEL); }, nullptr,
          [](bool gpu) { return std::make_shared<TCudaBlockEquivalence3D>(gpu, BE_ALGO_PIXEL); }}},
        {"runeq",
         {"Run equivalence by Bekhtin et.al. 2015 (4-connected, B200)", nullptr,
          [](bool gpu) { return std::make_shared<TCudaRunEquivalence>(gpu); }, nullptr, nullptr}},
    };
    return list;
}

std::shared_ptr<ILabeling> SetLabelingAlg(const std::string &name, bool useGPU, bool label3D)
{
    auto it = AlgList().find(name);
    if (it == AlgList().end()) throw Error(BE_ERR_INVALID, "No labeling algorithm specified");
    const Algs &a = it->second;
    std::shared_ptr<ILabeling> alg;
    if (!label3D) alg = useGPU ? (a.gpu ? a.gpu(true) : nullptr) : (a.cpu ? a.cpu() : nullptr);
    else alg = useGPU ? (a.gpu3d ? a.gpu3d(true) : nullptr) : (a.cpu3d ? a.cpu3d() : nullptr);
    if (!alg) throw Error(BE_ERR_INVALID, "Chosen algorithm doesn't support specified capabilities");
    return alg;
}

}  // namespace LabelingB200

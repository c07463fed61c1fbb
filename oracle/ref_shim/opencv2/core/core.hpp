// Minimal stand-in for <opencv2/core/core.hpp>: the part of cv::Mat that the reference's labeling
// sources use (2D and 3D dense matrices of 8-bit or 32-bit single-channel elements, shallow copies
// sharing one buffer, ROI views, at<>, zeros, copyTo).  Written from OpenCV's public API semantics.
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef signed char schar;

#define CV_8U 0
#define CV_32S 4
#define CV_CN_SHIFT 3
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << CV_CN_SHIFT))
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32SC1 CV_MAKETYPE(CV_32S, 1)

namespace cv {

struct Scalar {
    double v0;
    Scalar(double v = 0) : v0(v) {}
};

struct Size {
    int width, height;
    Size(int w = 0, int h = 0) : width(w), height(h) {}
};

struct Rect {
    int x, y, width, height;
    Rect(int x_ = 0, int y_ = 0, int w = 0, int h = 0) : x(x_), y(y_), width(w), height(h) {}
};

struct MatSize {
    const int *p;
    int operator[](int i) const { return p[i]; }
    operator const int *() const { return p; }
};

class Mat {
public:
    int dims = 0, rows = 0, cols = 0;
    uchar *data = nullptr;
    size_t step[3] = {0, 0, 0};   // bytes between consecutive indices of each dimension
    int sz[3] = {0, 0, 0};
    MatSize size{sz};

    Mat() = default;
    Mat(int r, int c, int type) { create2(r, c, type); }
    Mat(int r, int c, int type, const Scalar &s) { create2(r, c, type); fill(s); }
    Mat(Size s, int type) { create2(s.height, s.width, type); }
    Mat(int nd, const int *sizes, int type, const Scalar &s = Scalar()) { createN(nd, sizes, type); fill(s); }
    Mat(const Mat &o) { *this = o; }
    Mat &operator=(const Mat &o)
    {
        dims = o.dims; rows = o.rows; cols = o.cols; data = o.data; type_ = o.type_; buf_ = o.buf_;
        for (int i = 0; i < 3; ++i) { step[i] = o.step[i]; sz[i] = o.sz[i]; }
        size.p = sz;
        return *this;
    }

    static Mat zeros(int r, int c, int type) { return Mat(r, c, type, Scalar(0)); }
    static Mat zeros(int nd, const int *sizes, int type) { return Mat(nd, sizes, type, Scalar(0)); }

    bool empty() const { return data == nullptr || total() == 0; }
    int type() const { return type_; }
    int depth() const { return type_ & 7; }
    int channels() const { return (type_ >> CV_CN_SHIFT) + 1; }
    size_t elemSize() const { return size_t(depth() == CV_32S ? 4 : 1) * channels(); }
    size_t total() const
    {
        size_t t = 1;
        for (int i = 0; i < dims; ++i) t *= size_t(sz[i]);
        return dims ? t : 0;
    }
    bool isContinuous() const { return dims != 2 || step[0] == size_t(cols) * elemSize(); }

    template <class T> T &at(int i, int j) { return *reinterpret_cast<T *>(data + i * step[0] + j * step[1]); }
    template <class T> const T &at(int i, int j) const
    {
        return *reinterpret_cast<const T *>(data + i * step[0] + j * step[1]);
    }
    template <class T> T &at(int i, int j, int k)
    {
        return *reinterpret_cast<T *>(data + i * step[0] + j * step[1] + k * step[2]);
    }
    template <class T> const T &at(int i, int j, int k) const
    {
        return *reinterpret_cast<const T *>(data + i * step[0] + j * step[1] + k * step[2]);
    }

    // ROI view sharing this matrix's buffer (2D only).
    Mat operator()(const Rect &r) const
    {
        Mat m(*this);
        m.data = data + r.y * step[0] + r.x * step[1];
        m.rows = m.sz[0] = r.height;
        m.cols = m.sz[1] = r.width;
        return m;
    }

    void copyTo(Mat &dst) const
    {
        if (dst.empty() || dst.type_ != type_ || dst.total() != total()) {
            if (dims == 2) dst.create2(rows, cols, type_);
            else dst.createN(dims, sz, type_);
        }
        copyInto(dst);
    }
    void copyTo(Mat &&dst) const { copyInto(dst); }   // into an existing view of the same size

private:
    int type_ = 0;
    std::shared_ptr<std::vector<uchar>> buf_;

    void create2(int r, int c, int type)
    {
        const int s[2] = {r, c};
        createN(2, s, type);
    }
    void createN(int nd, const int *sizes, int type)
    {
        type_ = type;
        dims = nd;
        for (int i = 0; i < 3; ++i) sz[i] = i < nd ? sizes[i] : 0;
        size.p = sz;
        rows = sz[0];
        cols = nd > 1 ? sz[1] : 1;
        size_t s = elemSize();
        for (int i = nd - 1; i >= 0; --i) { step[i] = s; s *= size_t(sz[i]); }
        // Zeroed slack past the end: the reference's block labelers read up to two rows past the
        // last one at an even-height bottom border (LabelingAlgs.cpp:366-374, 396-399).
        const size_t slack = (nd == 2 ? 2 * step[0] : 0) + 64;
        buf_ = std::make_shared<std::vector<uchar>>(s + slack);
        data = buf_->data();
    }
    void fill(const Scalar &s)
    {
        const size_t n = total();
        if (depth() == CV_32S) {
            int32_t *p = reinterpret_cast<int32_t *>(data);
            for (size_t i = 0; i < n * channels(); ++i) p[i] = int32_t(s.v0);
        } else {
            memset(data, int(s.v0), n * channels());
        }
    }
    void copyInto(Mat &dst) const
    {
        if (dims != 2) {
            memcpy(dst.data, data, total() * elemSize());
            return;
        }
        const size_t row_bytes = size_t(cols) * elemSize();
        for (int r = 0; r < rows; ++r) memcpy(dst.data + r * dst.step[0], data + r * step[0], row_bytes);
    }
};

}  // namespace cv

// Minimal stand-in for the OpenCV 1.x C API header, enough for the reference's vendored Grana
// labeler (Labeling2015/src/cvlabeling_imagelab.cpp) to compile, and for LabelingAlgs.cpp's
// IplImage(cv::Mat) conversion when REF_SHIM_IPL_FROM_MAT is defined.  TEST INFRASTRUCTURE ONLY.
#pragma once
#ifdef REF_SHIM_IPL_FROM_MAT
#include "../opencv2/core/core.hpp"
#endif
typedef struct _IplImage {
    int width, height, widthStep;
    char *imageData;
#ifdef REF_SHIM_IPL_FROM_MAT
    _IplImage(int w, int h, int ws, char *d) : width(w), height(h), widthStep(ws), imageData(d) {}
    _IplImage(const cv::Mat &m)
        : width(m.cols), height(m.rows), widthStep(int(m.step[0])), imageData(reinterpret_cast<char *>(m.data)) {}
#endif
} IplImage;
#define CVAPI(rettype) extern "C" rettype
#define CV_IMPL extern "C"
#define CV_FUNCNAME(name)

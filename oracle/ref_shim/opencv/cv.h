// Minimal stand-in for the OpenCV 1.x C API header, enough for the reference's vendored Grana
// labeler (Labeling2015/src/cvlabeling_imagelab.cpp) to compile.  TEST INFRASTRUCTURE ONLY.
#pragma once
typedef struct _IplImage {
    int width, height, widthStep;
    char *imageData;
} IplImage;
#define CVAPI(rettype) extern "C" rettype
#define CV_IMPL extern "C"
#define CV_FUNCNAME(name)

// Minimal stand-in for <opencv2/imgproc/imgproc.hpp>: the three calls the reference's labeling
// sources name.  threshold() has OpenCV's THRESH_BINARY meaning (dst = src > thresh ? maxval : 0);
// the others are defined in ref_cpu.cpp and are not used on the timed path.
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "../core/core.hpp"

namespace cv {
enum { COLOR_RGB2GRAY = 7 };
enum { THRESH_BINARY = 0, THRESH_OTSU = 8 };
void cvtColor(const Mat &src, Mat &dst, int code);
double threshold(const Mat &src, Mat &dst, double thresh, double maxval, int type);
int connectedComponents(const Mat &src, Mat &labels, int connectivity, int ltype);
}  // namespace cv

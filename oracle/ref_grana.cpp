// ref_grana.cpp -- C entry point around the reference's vendored Grana block labeler
// (Labeling2015/src/cvlabeling_imagelab.cpp, compiled in place from the reference tree by
// oracle/Makefile into oracle/_ref/libref_grana.so).  TEST INFRASTRUCTURE ONLY: a second oracle for
// 8-connected 2D labeling and a timed CPU baseline.
//
// TBlockGranaLabeling::DoLabel (Labeling2015/src/LabelingAlgs.cpp:51-57) calls
// cvLabelingImageLab(src, dst, 255, &n) on the binarized image.  icvLabelImage sizes its label
// tables as w*h/4 ints (cvlabeling_imagelab.cpp:54-56) while it can create up to
// ceil(w/2)*ceil(h/2) labels (1-based), which overruns for odd sizes and for images whose every
// 2x2 block starts a new label.  This wrapper therefore hands it an image extended by zero rows to
// an even width and at least two extra rows, which only enlarges the tables; labels of the
// original pixels are unchanged.
#include <opencv/cv.h>

#include <cstdint>
#include <cstring>
#include <vector>

extern "C" void cvLabelingImageLab(IplImage *srcImage, IplImage *dstImage,
                                   unsigned char byForeground, int *numLabels);

extern "C" int ref_grana(const uint8_t *img, long rows, long cols, long pitch, int thr,
                         int32_t *out, int *num_labels)
{
    if (rows <= 0 || cols <= 0) return -1;
    const long w = (cols + 1) & ~1L, h = ((rows + 1) & ~1L) + 2;
    std::vector<uint8_t> src((size_t)w * h, 0);
    std::vector<int32_t> dst((size_t)w * h, 0);
    for (long y = 0; y < rows; ++y)
        for (long x = 0; x < cols; ++x) src[(size_t)y * w + x] = img[y * pitch + x] > thr ? 255 : 0;
    IplImage s{(int)w, (int)h, (int)w, (char *)src.data()};
    IplImage d{(int)w, (int)h, (int)(w * 4), (char *)dst.data()};
    int n = 0;
    cvLabelingImageLab(&s, &d, 255, &n);
    for (long y = 0; y < rows; ++y) std::memcpy(out + y * cols, dst.data() + (size_t)y * w, 4 * cols);
    if (num_labels) *num_labels = n;
    return 0;
}

// Minimal stand-in for the OpenCV C++ header, written for this project so that the
// reference program (zhangyuyi99/cuda_multiDDM, src/DDM.cu and src/video_reader.cpp)
// compiles without OpenCV. It declares only the cv:: names those two files use.
//
// The reference is only ever run here in its benchmark (-B) and .movie (-M) input
// modes, which never touch a capture object. Every capture or display operation in
// this stub therefore prints a message and exits with status 1: a run that reaches
// one of them is a run this build cannot serve.
#ifndef DDM_ORACLE_OPENCV_STUB_HPP
#define DDM_ORACLE_OPENCV_STUB_HPP

#include <cstdio>
#include <cstdlib>
#include <string>

namespace cv {

[[noreturn]] inline void stub_unavailable(const char *what) {
    std::fprintf(stderr, "[opencv stub] %s is unavailable in this build\n", what);
    std::exit(1);
}

enum { CAP_PROP_FPS = 5, CAP_PROP_FRAME_WIDTH = 3, CAP_PROP_FRAME_HEIGHT = 4 };

struct Scalar {
    double v[4];
    Scalar(double a = 0, double b = 0, double c = 0, double d = 0) : v{a, b, c, d} {}
};

struct Rect {
    int x, y, width, height;
    Rect(int x_, int y_, int w_, int h_) : x(x_), y(y_), width(w_), height(h_) {}
};

struct Mat {
    int rows = 0, cols = 0;
    size_t step = 0;
    unsigned char *data = nullptr;
    int type() const { return 0; }
    int depth() const { return 0; }
    int channels() const { return 1; }
    bool empty() const { return true; }
    bool isContinuous() const { return true; }
    size_t elemSize() const { return 1; }
    size_t elemSize1() const { return 1; }
    template <typename T> T &at(int, int) { stub_unavailable("cv::Mat::at"); }
};

struct VideoCapture {
    VideoCapture() {}
    explicit VideoCapture(int) { stub_unavailable("cv::VideoCapture(camera)"); }
    explicit VideoCapture(const std::string &) { stub_unavailable("cv::VideoCapture(file)"); }
    bool isOpened() const { return false; }
    double get(int) const { stub_unavailable("cv::VideoCapture::get"); }
    void release() {}
    VideoCapture &operator>>(Mat &) { stub_unavailable("cv::VideoCapture::read"); }
};

inline void rectangle(Mat &, const Rect &, const Scalar &) { stub_unavailable("cv::rectangle"); }
inline void imshow(const std::string &, const Mat &) { stub_unavailable("cv::imshow"); }
inline int waitKey(int) { stub_unavailable("cv::waitKey"); }
inline void destroyAllWindows() {}

}  // namespace cv

#endif

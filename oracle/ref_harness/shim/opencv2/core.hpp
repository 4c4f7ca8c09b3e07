// Test-only stand-in for the handful of cv::Mat members that the reference's
// shared data-model header and PatchMatch translation unit touch (rows, cols,
// data, ptr<T>(row), at<T>(row, col), empty()).  It exists so the reference's
// own patchmatch_mvs.cu compiles unmodified for the GPU reference harness.
#pragma once
#include <cstddef>
#include <cstring>
#include <memory>
#include <vector>

#define CV_8U 0
#define CV_32F 5
#define CV_64F 6
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << 3))
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)

namespace cv {

struct Scalar {
    double v0;
    Scalar(double a = 0.0) : v0(a) {}
};

struct KeyPoint {
    float x = 0, y = 0, size = 0, angle = 0, response = 0;
    int octave = 0, class_id = -1;
};

class Mat {
public:
    int rows = 0, cols = 0;
    int type_ = 0;
    unsigned char* data = nullptr;

    Mat() = default;
    Mat(int r, int c, int t) { create(r, c, t); }
    Mat(int r, int c, int t, const Scalar& s) {
        create(r, c, t);
        if ((t & 7) == CV_32F) {
            float* p = reinterpret_cast<float*>(data);
            for (size_t i = 0; i < total() * channels(); ++i) p[i] = static_cast<float>(s.v0);
        }
    }

    void create(int r, int c, int t) {
        rows = r; cols = c; type_ = t;
        buf_ = std::make_shared<std::vector<unsigned char>>(total() * elemSize());
        data = buf_->data();
    }

    bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
    size_t total() const { return static_cast<size_t>(rows) * cols; }
    int channels() const { return ((type_ >> 3) & 511) + 1; }
    size_t elemSize1() const {
        switch (type_ & 7) { case CV_8U: return 1; case CV_32F: return 4; case CV_64F: return 8; }
        return 4;
    }
    size_t elemSize() const { return elemSize1() * channels(); }
    int type() const { return type_; }

    template <typename T> T* ptr(int r) { return reinterpret_cast<T*>(data + r * cols * elemSize()); }
    template <typename T> const T* ptr(int r) const { return reinterpret_cast<const T*>(data + r * cols * elemSize()); }
    template <typename T> T& at(int r, int c) { return ptr<T>(r)[c]; }
    template <typename T> const T& at(int r, int c) const { return ptr<T>(r)[c]; }

private:
    std::shared_ptr<std::vector<unsigned char>> buf_;
};

}  // namespace cv

// TEST INFRASTRUCTURE ONLY.  A minimal stand-in for the part of OpenCV that
// the reference's hot-path sources touch: a reference-counted 2-D matrix of
// 8U / 32S / 32F single-channel elements (cv::Mat with at<T>, zeros, ones,
// size, type, clone and a borrowed-data constructor), cv::Size, cv::Scalar,
// and cv::resize of single-channel masks.  Written for this project from
// OpenCV's documented behaviour; it is not OpenCV source.  Used only to
// compile the reference's sources into oracle/_ref.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

typedef unsigned char uchar;

// element types, as OpenCV's global macros
#define CV_8U 0
#define CV_32S 4
#define CV_32F 5
#define CV_8UC1 0
#define CV_32SC1 4
#define CV_32FC1 5
#define CV_8UC3 16

namespace cv {

using ::uchar;

enum { INTER_NEAREST = 0, INTER_LINEAR = 1, INTER_AREA = 3 };
enum { MORPH_RECT = 0, MORPH_CROSS = 1, MORPH_ELLIPSE = 2 };

inline size_t elem_size(int type) { return type == CV_8UC1 ? 1 : type == CV_8UC3 ? 3 : 4; }

struct Size {
  int width = 0, height = 0;
  Size() {}
  Size(int w, int h) : width(w), height(h) {}
  bool operator==(const Size& o) const { return width == o.width && height == o.height; }
  bool operator!=(const Size& o) const { return !(*this == o); }
};
inline Size operator/(const Size& s, int d) { return Size(s.width / d, s.height / d); }
inline Size operator*(const Size& s, int m) { return Size(s.width * m, s.height * m); }

template <typename T, int N> struct Vec {
  T v[N];
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};
typedef Vec<uchar, 3> Vec3b;

struct Scalar {
  double v0 = 0;
  Scalar() {}
  Scalar(double v) : v0(v) {}
};

class Mat {
  std::shared_ptr<std::vector<uchar>> own_;
  int type_ = CV_8UC1;

  void alloc(int r, int c, int t) {
    rows = r; cols = c; type_ = t;
    own_ = std::make_shared<std::vector<uchar>>((size_t)r * c * elem_size(t));
    data = own_->data();
  }
  template <typename T> void fill(double v) {
    T* p = (T*)data;
    for (size_t i = 0; i < (size_t)rows * cols; ++i) p[i] = (T)v;
  }
  void fill_scalar(double v) {
    if (type_ == CV_8UC3) { for (size_t i = 0; i < 3 * total(); ++i) data[i] = (uchar)v; return; }
    if (type_ == CV_8UC1) fill<uchar>(v); else if (type_ == CV_32SC1) fill<int32_t>(v); else fill<float>(v);
  }

 public:
  int rows = 0, cols = 0;
  uchar* data = nullptr;

  Mat() {}
  Mat(int r, int c, int t) { alloc(r, c, t); }
  Mat(Size s, int t) { alloc(s.height, s.width, t); }
  Mat(int r, int c, int t, const Scalar& v) { alloc(r, c, t); fill_scalar(v.v0); }
  Mat(Size s, int t, const Scalar& v) { alloc(s.height, s.width, t); fill_scalar(v.v0); }
  // borrowed caller storage, as OpenCV's Mat(rows, cols, type, data)
  Mat(int r, int c, int t, void* p) : type_(t), rows(r), cols(c), data((uchar*)p) {}
  Mat(Size s, int t, void* p) : type_(t), rows(s.height), cols(s.width), data((uchar*)p) {}

  static Mat zeros(int r, int c, int t) { return Mat(r, c, t, Scalar(0)); }
  static Mat zeros(Size s, int t) { return Mat(s, t, Scalar(0)); }
  static Mat ones(int r, int c, int t) { return Mat(r, c, t, Scalar(1)); }
  static Mat ones(Size s, int t) { return Mat(s, t, Scalar(1)); }

  int type() const { return type_; }
  int depth() const { return type_; }
  int channels() const { return 1; }
  size_t elemSize() const { return elem_size(type_); }
  size_t total() const { return (size_t)rows * cols; }
  bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
  Size size() const { return Size(cols, rows); }
  Mat clone() const {
    Mat m(rows, cols, type_);
    if (!empty()) std::memcpy(m.data, data, total() * elemSize());
    return m;
  }
  void create(int r, int c, int t) { if (rows != r || cols != c || type_ != t || !data) alloc(r, c, t); }
  void create(Size s, int t) { create(s.height, s.width, t); }
  template <typename T> T& at(int r, int c) { return ((T*)data)[(size_t)r * cols + c]; }
  template <typename T> const T& at(int r, int c) const { return ((const T*)data)[(size_t)r * cols + c]; }
  template <typename T> T& at(int i) { return ((T*)data)[i]; }
  template <typename T> const T& at(int i) const { return ((const T*)data)[i]; }
  template <typename T> T* ptr(int r = 0) { return (T*)data + (size_t)r * cols; }
  template <typename T> const T* ptr(int r = 0) const { return (const T*)data + (size_t)r * cols; }
};

// resize of a single-channel 8U mask.  An exact halving is an area average
// (OpenCV's INTER_LINEAR switches to INTER_AREA for integer 2x downscales),
// rounded to nearest; any other factor samples bilinearly at
// (x + 0.5) * scale - 0.5, rounded to nearest (for the 4x case the two taps
// per axis weigh 1/2 each, which OpenCV's 11-bit fixed point also represents
// exactly).
inline void resize(const Mat& src, Mat& dst, Size ds, double = 0, double = 0, int = INTER_LINEAR) {
  Mat out(ds, src.type());
  const int sw = src.cols, sh = src.rows;
  for (int y = 0; y < ds.height; ++y)
    for (int x = 0; x < ds.width; ++x) {
      double v;
      if (sw == 2 * ds.width && sh == 2 * ds.height) {
        double s = 0;
        for (int dy = 0; dy < 2; ++dy)
          for (int dx = 0; dx < 2; ++dx)
            s += src.type() == CV_8UC1 ? src.at<uchar>(2 * y + dy, 2 * x + dx) : src.at<float>(2 * y + dy, 2 * x + dx);
        v = s / 4;
      } else {
        const double fx = (x + 0.5) * sw / ds.width - 0.5, fy = (y + 0.5) * sh / ds.height - 0.5;
        int x0 = (int)std::floor(fx), y0 = (int)std::floor(fy);
        double ax = fx - x0, ay = fy - y0;
        auto px = [&](int yy, int xx) -> double {
          xx = xx < 0 ? 0 : (xx >= sw ? sw - 1 : xx);
          yy = yy < 0 ? 0 : (yy >= sh ? sh - 1 : yy);
          return src.type() == CV_8UC1 ? (double)src.at<uchar>(yy, xx) : (double)src.at<float>(yy, xx);
        };
        v = px(y0, x0) * (1 - ax) * (1 - ay) + px(y0, x0 + 1) * ax * (1 - ay) +
            px(y0 + 1, x0) * (1 - ax) * ay + px(y0 + 1, x0 + 1) * ax * ay;
      }
      if (src.type() == CV_8UC1) out.at<uchar>(y, x) = (uchar)std::floor(v + 0.5);
      else out.at<float>(y, x) = (float)v;
    }
  dst = out;
}

// image files are not written by the oracle (the reference writes them only
// in its debug paths)
inline bool imwrite(const std::string&, const Mat&) { return false; }

}  // namespace cv

// TEST INFRASTRUCTURE ONLY.  Minimal stand-in for the one OpenCV type the
// reference's SDF hot-path headers touch: a borrowed row-major float/uchar
// matrix read through at<T>(row, col).  Written for this project; it is not
// OpenCV source.  Used only to compile the reference headers into oracle/_ref.
#pragma once
#include <cstddef>
namespace cv {
struct Mat {
  int rows = 0, cols = 0;
  size_t elem = 4;
  unsigned char* data = nullptr;
  Mat() {}
  Mat(int r, int c, size_t e, void* p) : rows(r), cols(c), elem(e), data((unsigned char*)p) {}
  template <typename T> T& at(int r, int c) { return ((T*)data)[(size_t)r * cols + c]; }
  template <typename T> const T& at(int r, int c) const { return ((const T*)data)[(size_t)r * cols + c]; }
};
}  // namespace cv

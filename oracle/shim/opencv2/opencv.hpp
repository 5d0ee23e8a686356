/*
 * Stand-in for the small part of OpenCV's C++ API that the reference's fusion
 * sources use on the depth-fusion path (src/fusion/geometryfusion_mipmap_cpu.cpp,
 * mesh*.cpp, treeandbrick*.cpp).  ORACLE INFRASTRUCTURE ONLY: it lets the
 * unmodified reference sources compile into oracle/_ref/ so they can serve as
 * the checker and as the timed CPU baseline.  It is never part of the product.
 *
 * cv::Mat here is a plain reference-counted row-major buffer.  Only what the
 * fusion path touches is real (data/rows/cols/step/at<>/clone/copyTo/ptr);
 * image I/O and display are no-ops.
 */
#ifndef FF_ORACLE_SHIM_OPENCV_HPP
#define FF_ORACLE_SHIM_OPENCV_HPP

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <cmath>
#include <string>
#include <vector>
#include <deque>
#include <map>
#include <list>
#include <set>
#include <memory>
#include <algorithm>
#include <iostream>
#include <sstream>
#include <limits>
#include <cfloat>
#include <time.h>

typedef unsigned char uchar;
typedef unsigned short ushort;

#define CV_8U 0
#define CV_8S 1
#define CV_16U 2
#define CV_16S 3
#define CV_32S 4
#define CV_32F 5
#define CV_64F 6
#define CV_CN_SHIFT 3
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn)-1) << CV_CN_SHIFT))
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_8UC4 CV_MAKETYPE(CV_8U, 4)
#define CV_16UC1 CV_MAKETYPE(CV_16U, 1)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#define CV_32FC4 CV_MAKETYPE(CV_32F, 4)
#define CV_16UC3 CV_MAKETYPE(CV_16U, 3)
#define CV_64FC1 CV_MAKETYPE(CV_64F, 1)

namespace cv {

inline int shimElemSize1(int depth) {
  static const int s[] = {1, 1, 2, 2, 4, 4, 8, 8};
  return s[depth & 7];
}

template <typename T> struct DataType;
template <> struct DataType<double> { enum { type = CV_64FC1 }; };
template <> struct DataType<float> { enum { type = CV_32FC1 }; };
template <> struct DataType<uchar> { enum { type = CV_8UC1 }; };
template <> struct DataType<ushort> { enum { type = CV_16UC1 }; };

struct Size {
  int width, height;
  Size(int w = 0, int h = 0) : width(w), height(h) {}
};

struct Range {
  int start, end;
  Range(int s = 0, int e = 0) : start(s), end(e) {}
};

class Mat {
 public:
  int rows, cols, flags;
  uchar *data;
  size_t step;
  std::shared_ptr<std::vector<uchar> > store;

  Mat() : rows(0), cols(0), flags(0), data(NULL), step(0) {}
  Mat(int r, int c, int type) { create(r, c, type); }
  Mat(Size s, int type) { create(s.height, s.width, type); }
  Mat(int r, int c, int type, void *ext, size_t st = 0)
      : rows(r), cols(c), flags(type), data((uchar *)ext) {
    step = st ? st : (size_t)c * elemSize();
  }
  void create(int r, int c, int type) {
    rows = r;
    cols = c;
    flags = type;
    step = (size_t)c * elemSize();
    store.reset(new std::vector<uchar>((size_t)r * step + 32, 0));
    data = store->data();
  }
  int type() const { return flags; }
  int depth() const { return flags & 7; }
  int channels() const { return (flags >> CV_CN_SHIFT) + 1; }
  size_t elemSize() const { return (size_t)shimElemSize1(depth()) * channels(); }
  size_t elemSize1() const { return (size_t)shimElemSize1(depth()); }
  size_t total() const { return (size_t)rows * cols; }
  bool empty() const { return data == NULL || rows == 0 || cols == 0; }
  Size size() const { return Size(cols, rows); }
  template <typename T> T &at(int r, int c) { return *(T *)(data + (size_t)r * step + (size_t)c * sizeof(T)); }
  template <typename T> const T &at(int r, int c) const { return *(const T *)(data + (size_t)r * step + (size_t)c * sizeof(T)); }
  template <typename T> T &at(int i) { return ((T *)data)[i]; }
  template <typename T> const T &at(int i) const { return ((const T *)data)[i]; }
  uchar *ptr(int r = 0) { return data + (size_t)r * step; }
  const uchar *ptr(int r = 0) const { return data + (size_t)r * step; }
  template <typename T> T *ptr(int r = 0) { return (T *)(data + (size_t)r * step); }
  Mat clone() const {
    Mat m;
    if (!data) return m;
    m.create(rows, cols, flags);
    for (int r = 0; r < rows; r++) memcpy(m.ptr(r), ptr(r), (size_t)cols * elemSize());
    return m;
  }
  void copyTo(Mat &m) const { m = clone(); }
  void release() { store.reset(); data = NULL; rows = cols = 0; }
  void convertTo(Mat &m, int, double = 1.0, double = 0.0) const { m = clone(); }
  Mat t() const { return clone(); }
  Mat inv() const { return clone(); }
  Mat row(int) const { return clone(); }
  Mat col(int) const { return clone(); }
  Mat rowRange(int, int) const { return clone(); }
  Mat colRange(int, int) const { return clone(); }
  Mat operator()(Range, Range) const { return clone(); }
  Mat &operator*=(double) { return *this; }
  Mat &setTo(double, bool = false) { return *this; }
  static Mat eye(int r, int c, int type) {
    Mat m(r, c, type);
    for (int i = 0; i < r && i < c; i++) m.at<double>(i, i) = 1.0;
    return m;
  }
  static Mat zeros(int r, int c, int type) { return Mat(r, c, type); }
  template <typename T> operator std::vector<T>() const {
    return std::vector<T>((const T *)data, (const T *)data + total() * channels());
  }
};

inline Mat operator*(const Mat &a, const Mat &) { return a.clone(); }
inline Mat operator-(const Mat &a) { return a.clone(); }
inline Mat operator+(const Mat &a, const Mat &) { return a.clone(); }
inline Mat operator-(const Mat &a, double) { return a.clone(); }
inline Mat operator*(const Mat &a, double) { return a.clone(); }
inline Mat operator/(const Mat &a, double) { return a.clone(); }
inline bool operator==(const Mat &, double) { return false; }

inline int64_t getTickCount() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (int64_t)ts.tv_sec * 1000000000LL + ts.tv_nsec;
}
inline double getTickFrequency() { return 1e9; }
inline Mat imread(const std::string &, int = 1) { return Mat(); }
inline bool imwrite(const std::string &, const Mat &) { return true; }
inline void imshow(const std::string &, const Mat &) {}
inline int waitKey(int = 0) { return -1; }
inline void split(const Mat &, std::vector<Mat> &) {}
inline void merge(const std::vector<Mat> &, Mat &) {}

}  // namespace cv

#endif

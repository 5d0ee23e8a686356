/*
 * CameraInfo / Frustum for the reference's camerautils.hpp interface, in plain
 * double arithmetic.  ORACLE INFRASTRUCTURE ONLY: the reference's own
 * camerautils.cpp needs Eigen and OpenCV, neither of which is installed, so
 * the oracle build links this file in its place.
 *
 * Semantics follow the reference (src/camerautils/camerautils.cpp):
 *  - the extrinsic [R|t] maps camera to world coordinates;
 *  - getExtrinsicInverse() returns [R^T | -R^T t] (camerautils.cpp:153-161);
 *  - setExtrinsic() takes R from the upper-left 3x3 block and t from column 3.
 * The products are summed left to right, ((a0*b0 + a1*b1) + a2*b2), the order
 * of a naive 3x3 GEMM; the product path computes the pose with the same order.
 */
#include <camerautils/camerautils.hpp>

CameraInfo::CameraInfo(const cv::Mat &, int decompositionMethod)
    : _intrinsic(cv::Mat::eye(3, 3, CV_64FC1)),
      _rotation(cv::Mat::eye(3, 3, CV_64FC1)),
      _translation(cv::Mat::zeros(3, 1, CV_64FC1)),
      _decompositionMethod(decompositionMethod) {}

CameraInfo::CameraInfo(const CameraInfo &info)
    : _intrinsic(info._intrinsic.clone()),
      _rotation(info._rotation.clone()),
      _translation(info._translation.clone()),
      _decompositionMethod(info._decompositionMethod) {}

CameraInfo::~CameraInfo() {}

CameraInfo &CameraInfo::operator=(const CameraInfo &info) {
  _intrinsic = info._intrinsic.clone();
  _rotation = info._rotation.clone();
  _translation = info._translation.clone();
  _decompositionMethod = info._decompositionMethod;
  return *this;
}

bool CameraInfo::setIntrinsic(const cv::Mat &intrinsic) {
  _intrinsic = intrinsic.clone();
  return true;
}

bool CameraInfo::setExtrinsic(const cv::Mat &e) {
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) _rotation.at<double>(r, c) = e.at<double>(r, c);
    _translation.at<double>(r, 0) = e.at<double>(r, 3);
  }
  return true;
}

bool CameraInfo::setRotation(const cv::Mat &rotation) {
  _rotation = rotation.clone();
  return true;
}

bool CameraInfo::setRotationLogarithm(const cv::Mat &) { return false; }

void CameraInfo::setTranslation(const cv::Mat &translation) { _translation = translation.clone(); }

bool CameraInfo::setProjection(const cv::Mat &) { return false; }

cv::Mat CameraInfo::getIntrinsic() const { return _intrinsic.clone(); }
cv::Mat CameraInfo::getRotation() const { return _rotation.clone(); }
cv::Mat CameraInfo::getTranslation() const { return _translation.clone(); }

cv::Mat CameraInfo::getExtrinsic() const {
  cv::Mat m = cv::Mat::eye(4, 4, CV_64FC1);
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) m.at<double>(r, c) = _rotation.at<double>(r, c);
    m.at<double>(r, 3) = _translation.at<double>(r, 0);
  }
  return m;
}

cv::Mat CameraInfo::getExtrinsicInverse() const {
  cv::Mat m = cv::Mat::eye(4, 4, CV_64FC1);
  const cv::Mat &R = _rotation;
  const cv::Mat &t = _translation;
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) m.at<double>(r, c) = R.at<double>(c, r);
    double s = R.at<double>(0, r) * t.at<double>(0, 0) + R.at<double>(1, r) * t.at<double>(1, 0);
    s = s + R.at<double>(2, r) * t.at<double>(2, 0);
    m.at<double>(r, 3) = -s;
  }
  return m;
}

cv::Mat CameraInfo::getProjection() const { return cv::Mat::eye(3, 4, CV_64FC1); }
cv::Mat CameraInfo::getRotationQuaternion() const { return cv::Mat::zeros(4, 1, CV_64FC1); }
cv::Mat CameraInfo::getRotationLogarithm() const { return cv::Mat::zeros(3, 1, CV_64FC1); }
cv::Mat CameraInfo::getQuaternion() const { return cv::Mat::zeros(4, 1, CV_64FC1); }
void CameraInfo::scale(double) {}
void CameraInfo::projectTo(CameraInfo, cv::Mat &, cv::Mat &) {}
bool CameraInfo::decomposeAndFixProjectionMatrixOpenCV(const cv::Mat &, cv::Mat &, cv::Mat &, cv::Mat &) {
  return false;
}
void CameraInfo::CalculateRotation(double &, double &, double &, double &) const {}

Frustum::Frustum(float p_lx, float p_ly, float p_lz, float p_lo, float p_rx, float p_ry, float p_rz, float p_ro,
                 float p_tx, float p_ty, float p_tz, float p_to, float p_bx, float p_by, float p_bz, float p_bo,
                 float p_fx, float p_fy, float p_fz, float p_fo)
    : lx(p_lx), ly(p_ly), lz(p_lz), lo(p_lo), rx(p_rx), ry(p_ry), rz(p_rz), ro(p_ro), tx(p_tx), ty(p_ty),
      tz(p_tz), to(p_to), bx(p_bx), by(p_by), bz(p_bz), bo(p_bo), fx(p_fx), fy(p_fy), fz(p_fz), fo(p_fo) {}

/* The frustum is only computed on the float-depth addMap path, which the
 * oracle never runs; an all-accepting frustum keeps the link complete. */
Frustum::Frustum(const CameraInfo &, float, float, float)
    : lx(0), ly(0), lz(0), lo(-1e30f), rx(0), ry(0), rz(0), ro(-1e30f), tx(0), ty(0), tz(0), to(-1e30f), bx(0),
      by(0), bz(0), bo(-1e30f), fx(0), fy(0), fz(0), fo(-1e30f) {}

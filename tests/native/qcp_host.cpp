// Host build of the library's QCP header for CPU unit tests (test-only; the
// library itself runs this code on the device).
#include "qcp.cuh"

extern "C" {
double t_qcp_lambda(const double* h, double e0, int* iters, int* fallback) {
  wmd::QcpOut o = wmd::qcp_lambda(h, e0);
  if (iters) *iters = o.iters;
  if (fallback) *fallback = o.fallback;
  return o.lambda;
}
double t_lambda_svd(const double* h) { return wmd::lambda_from_svd(h); }
void t_rotation_qcp(const double* h, double lambda, double* r) { wmd::rotation_from_qcp(h, lambda, r); }
void t_rotation_svd(const double* h, double* r) { wmd::rotation_from_svd(h, r); }
// mixed-precision MSD of the tensor-core epilogue: 1 and *msd when accepted,
// 0 when the caller must take the FP64 route
int t_qcp_msd_mixed(const long long* h, double gx, double gy, float n, float s2, float* msd) {
  return wmd::qcp_msd_mixed(h, gx, gy, n, s2, msd) ? 1 : 0;
}
}

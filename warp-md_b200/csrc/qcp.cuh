// qcp.cuh -- FP64 optimal-superposition math shared by every kernel.
//
// Given the 3x3 cross-covariance H = sum_k (x_k - cx)(y_k - cy)^T of a frame x
// against a reference y, the minimum over rotations R of sum |R(x_k-cx) - (y_k-cy)|^2
// is G_x + G_y - 2 lambda_max, where lambda_max = s1 + s2 + sign(det H) s3 (s_i the
// singular values of H) is the largest eigenvalue of the 4x4 quaternion key
// matrix K(H) (Horn 1987).  The reference (warp-md plan.rs:1161-1248,
// math.rs:7-38) gets the same number from an nalgebra SVD with the
// reflection fix; this file uses QCP: Newton iteration on the characteristic
// polynomial of K (Theobald 2005, Acta Cryst A61:478-480; Liu, Agrafiotis &
// Theobald 2010, J Comput Chem 31:1561), in FP64, starting from the upper
// bound (G_x + G_y)/2.  When the largest root is (nearly) double -- collinear or
// planar structures -- the polynomial route loses accuracy, so lambda is then
// taken from a one-sided Jacobi SVD (Hestenes 1958) instead.
//
// The rotation (needed by the gradient) is re-derived from the eigenvector of
// K for lambda_max, read off the adjugate of (K - lambda I), and converted to
// the rotation matrix that maps frame coordinates onto the reference
// (the same R = V U^T the reference builds).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define WMD_HD __host__ __device__ __forceinline__
#else
#define WMD_HD inline
#endif

namespace wmd {

WMD_HD double det3(const double m[9]) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// Key matrix K (row-major 4x4, symmetric) of H (row-major, H[a][b] = sum x_a y_b).
WMD_HD void key_matrix(const double h[9], double k[16]) {
  const double sxx = h[0], sxy = h[1], sxz = h[2];
  const double syx = h[3], syy = h[4], syz = h[5];
  const double szx = h[6], szy = h[7], szz = h[8];
  k[0] = sxx + syy + szz; k[1] = syz - szy;        k[2] = szx - sxz;         k[3] = sxy - syx;
  k[4] = k[1];            k[5] = sxx - syy - szz;  k[6] = sxy + syx;         k[7] = szx + sxz;
  k[8] = k[2];            k[9] = k[6];             k[10] = -sxx + syy - szz; k[11] = syz + szy;
  k[12] = k[3];           k[13] = k[7];            k[14] = k[11];            k[15] = -sxx - syy + szz;
}

// Determinant of a 4x4 matrix by 2x2 minors of the first two and last two rows.
WMD_HD double det4(const double k[16]) {
  const double s0 = k[0] * k[5] - k[1] * k[4];
  const double s1 = k[0] * k[6] - k[2] * k[4];
  const double s2 = k[0] * k[7] - k[3] * k[4];
  const double s3 = k[1] * k[6] - k[2] * k[5];
  const double s4 = k[1] * k[7] - k[3] * k[5];
  const double s5 = k[2] * k[7] - k[3] * k[6];
  const double c5 = k[10] * k[15] - k[11] * k[14];
  const double c4 = k[9] * k[15] - k[11] * k[13];
  const double c3 = k[9] * k[14] - k[10] * k[13];
  const double c2 = k[8] * k[15] - k[11] * k[12];
  const double c1 = k[8] * k[14] - k[10] * k[12];
  const double c0 = k[8] * k[13] - k[9] * k[12];
  return s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
}

// One-sided Jacobi SVD (Hestenes): returns singular values s (unsorted, >= 0)
// and, when u/v are non-null, the matching left/right singular vectors as
// columns (u column j = A v_j / s_j, left zero when s_j == 0).
WMD_HD void svd3_jacobi(const double a_in[9], double s[3], double* u, double* v) {
  double a[9];
  double vv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 9; ++i) a[i] = a_in[i];
  for (int sweep = 0; sweep < 40; ++sweep) {
    bool rotated = false;
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0;
      const int q = pq == 0 ? 1 : 2;
      double alpha = 0, beta = 0, gamma = 0;
      for (int r = 0; r < 3; ++r) {
        alpha += a[r * 3 + p] * a[r * 3 + p];
        beta += a[r * 3 + q] * a[r * 3 + q];
        gamma += a[r * 3 + p] * a[r * 3 + q];
      }
      if (gamma == 0.0 || fabs(gamma) <= 1e-17 * sqrt(alpha * beta)) continue;
      rotated = true;
      const double zeta = (beta - alpha) / (2.0 * gamma);
      const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
      const double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
      for (int r = 0; r < 3; ++r) {
        const double ap = a[r * 3 + p], aq = a[r * 3 + q];
        a[r * 3 + p] = c * ap - sn * aq;
        a[r * 3 + q] = sn * ap + c * aq;
        const double vp = vv[r * 3 + p], vq = vv[r * 3 + q];
        vv[r * 3 + p] = c * vp - sn * vq;
        vv[r * 3 + q] = sn * vp + c * vq;
      }
    }
    if (!rotated) break;
  }
  for (int j = 0; j < 3; ++j) {
    s[j] = sqrt(a[j] * a[j] + a[3 + j] * a[3 + j] + a[6 + j] * a[6 + j]);
    if (u) {
      const double inv = s[j] > 0 ? 1.0 / s[j] : 0.0;
      for (int r = 0; r < 3; ++r) u[r * 3 + j] = a[r * 3 + j] * inv;
    }
  }
  if (v)
    for (int i = 0; i < 9; ++i) v[i] = vv[i];
}

// lambda_max from the SVD: s1 + s2 + sign(det H) * s_min.
WMD_HD double lambda_from_svd(const double h[9]) {
  double s[3];
  svd3_jacobi(h, s, nullptr, nullptr);
  double smin = s[0];
  if (s[1] < smin) smin = s[1];
  if (s[2] < smin) smin = s[2];
  const double sum = s[0] + s[1] + s[2];
  return det3(h) < 0.0 ? sum - 2.0 * smin : sum;
}

#if defined(__CUDACC__)
// Device-side out-of-line SVD route, so that code paths that only rarely need
// it do not carry its registers.
__device__ __noinline__ inline double lambda_from_svd_call(const double* h) { return lambda_from_svd(h); }
#endif

struct QcpOut {
  double lambda;
  int iters;     // Newton iterations used
  int fallback;  // 1 when lambda came from the SVD
};

// Largest eigenvalue of K(H); e0 = (G_x + G_y) / 2 >= lambda_max.  The
// Newton step divides in IEEE FP64: on sm_100a that measured faster than a
// float reciprocal refined by FP64 Newton-Raphson steps.
WMD_HD QcpOut qcp_lambda(const double h[9], double e0) {
  QcpOut o{0.0, 0, 0};
  if (!(e0 > 0.0)) return o;
  double k[16];
  key_matrix(h, k);
  double c2 = 0.0;
  for (int i = 0; i < 9; ++i) c2 += h[i] * h[i];
  c2 *= -2.0;
  const double c1 = -8.0 * det3(h);
  const double c0 = det4(k);
  double l = e0;
  bool converged = false;
  int it = 0;
  for (; it < 60; ++it) {
    const double l2 = l * l;
    const double b = (l2 + c2) * l;
    const double a = b + c1;
    const double p = a * l + c0;               // P(l)  = l^4 + c2 l^2 + c1 l + c0
    const double dp = 2.0 * l2 * l + b + a;    // P'(l) = 4 l^3 + 2 c2 l + c1
    if (!(dp != 0.0)) break;
    const double delta = p / dp;
    l -= delta;
    if (fabs(delta) <= 1e-15 * fabs(l)) {
      converged = true;
      ++it;
      break;
    }
  }
  o.iters = it;
  // simple-root check: |P'(lambda)| = prod_{i>1} (lambda - lambda_i) is O(lambda^3)
  // unless another eigenvalue is within ~1e-6 relative of lambda_max.
  const double l3 = l * l * l;
  const double dp = 4.0 * l3 + 2.0 * c2 * l + c1;
  if (!converged || !(fabs(dp) > 1e-6 * 4.0 * fabs(l3)) || !(l == l)) {
#if defined(__CUDA_ARCH__)
    double tmp[9];  // only this rare branch takes an address
    for (int i = 0; i < 9; ++i) tmp[i] = h[i];
    o.lambda = lambda_from_svd_call(tmp);
#else
    o.lambda = lambda_from_svd(h);
#endif
    o.fallback = 1;
  } else {
    o.lambda = l;
  }
  return o;
}



// Mean-square deviation of a frame pair in the tensor-core epilogue, with as
// little FP64 arithmetic as the cancellation allows (on sm_100a FP64 issue
// stalls beside tensor-core MMAs, FP32 does not).  H (9 entries) is exact in
// integer units of s^2; gx, gy are the self-sums in the same units.  Written in
// u = 1 - lambda / e0 (e0 = (G_x + G_y) / 2 = D / 2, an upper bound of
// lambda_max), the characteristic polynomial of K divided by e0^4 is
//     Q(u) = det(M - u I) = u^4 - 4 u^3 + (6 + d2) u^2 - (4 + 2 d2 + d1) u + det(M),
// M = I - K / e0, d_k = c_k / e0^(4-k); its smallest root u1 = 1 - lambda_max / e0
// gives MSD = 2 e0 u1 / n.
//   * The constant term det(M) is where the cancellation sits (~8 u1 from O(1)
//     parts): M D = D I - 2K is formed from the exact inputs and its
//     determinant taken in FP64 (no division), then scaled by 1 / D^4 with an
//     FP32 reciprocal (a relative 1e-7 on this small term is harmless).
//   * The other coefficients are O(1) sums without cancellation (the roots
//     other than u1 lie near 1.3, so u1 is well conditioned) and are formed in
//     FP32 from H / e0.
//   * Newton from u = 0 runs in FP32, without FP64 divisions.
// Returns false, leaving *msd unset, when Newton did not converge to a clearly
// simple root (a second eigenvalue within ~1e-2 e0: collinear or nearly
// collinear structures); the caller then takes the FP64 route (qcp_lambda).
WMD_HD bool qcp_msd_mixed(const long long hq[9], double gx, double gy, float n, float s2, float* msd) {
  const double D = gx + gy;
  if (!(D > 0.0)) {
    *msd = 0.0f;
    return true;
  }
  const float invd = 1.0f / (float)D;
  // FP32 part first (fewer live registers): d2 = c2 / e0^2 = -2 sum h'^2,
  // d1 = c1 / e0^3 = -8 det h', h' = H / e0
  float b1, b2;
  {
    float hf[9];
    for (int i = 0; i < 9; ++i) hf[i] = (float)hq[i] * (2.0f * invd);
    float ss = 0.0f;
    for (int i = 0; i < 9; ++i) ss = fmaf(hf[i], hf[i], ss);
    const float det3f = hf[0] * (hf[4] * hf[8] - hf[5] * hf[7]) - hf[1] * (hf[3] * hf[8] - hf[5] * hf[6]) +
                        hf[2] * (hf[3] * hf[7] - hf[4] * hf[6]);
    const float d2 = -2.0f * ss, d1 = -8.0f * det3f;
    b1 = -(4.0f + 2.0f * d2 + d1);
    b2 = 6.0f + d2;
  }
  // M D = D I - 2 K (K as key_matrix, symmetric) from the exact inputs, in FP64
  const double h0 = (double)hq[0], h4 = (double)hq[4], h8 = (double)hq[8];
  const double m00 = D - 2.0 * (h0 + h4 + h8);
  const double m11 = D - 2.0 * (h0 - h4 - h8);
  const double m22 = D - 2.0 * (h4 - h0 - h8);
  const double m33 = D - 2.0 * (h8 - h0 - h4);
  const double h1 = (double)hq[1], h2 = (double)hq[2], h3 = (double)hq[3];
  const double h5 = (double)hq[5], h6 = (double)hq[6], h7 = (double)hq[7];
  const double m01 = -2.0 * (h5 - h7), m02 = -2.0 * (h6 - h2), m03 = -2.0 * (h1 - h3);
  const double m12 = -2.0 * (h1 + h3), m13 = -2.0 * (h6 + h2), m23 = -2.0 * (h5 + h7);
  // det of the symmetric M D by 2x2 minors of rows 2-3, then of rows 0-1 (as det4)
  const double c5 = m22 * m33 - m23 * m23, c4 = m12 * m33 - m23 * m13, c3 = m12 * m23 - m22 * m13;
  const double c2 = m02 * m33 - m23 * m03, c1 = m02 * m23 - m22 * m03, c0 = m02 * m13 - m12 * m03;
  double det = (m00 * m11 - m01 * m01) * c5;
  det -= (m00 * m12 - m02 * m01) * c4;
  det += (m00 * m13 - m03 * m01) * c3;
  det += (m01 * m12 - m02 * m11) * c2;
  det -= (m01 * m13 - m03 * m11) * c1;
  det += (m02 * m13 - m03 * m12) * c0;
  const double invd2 = (double)invd * (double)invd;  // D^-4 underflows FP32
  const float b0 = (float)(det * (invd2 * invd2));
  float u = 0.0f, dq = b1;
  bool converged = false;
  for (int it = 0; it < 24; ++it) {
    const float q = (((u - 4.0f) * u + b2) * u + b1) * u + b0;
    dq = ((4.0f * u - 12.0f) * u + 2.0f * b2) * u + b1;
    if (!(dq != 0.0f)) break;
    const float du = q / dq;
    u -= du;
    if (fabsf(du) <= 2e-7f * fabsf(u) + 1e-30f) {
      converged = true;
      break;
    }
  }
  dq = ((4.0f * u - 12.0f) * u + 2.0f * b2) * u + b1;
  // Near a double root (collinear or nearly collinear structures) the rounded
  // coefficients may carry no real root at all (the pair turns complex) and
  // Newton wanders; it only counts when it converged to a clearly simple root
  // (the slope there is ~2.4 for a well-spread structure).
  if (!converged || !(fabsf(dq) > 1e-2f) || !(u == u)) return false;
  const float mm = (float)D * u / n * s2;
  *msd = mm > 0.0f ? mm : 0.0f;
  return true;
}

// Mean-square deviation from the QCP eigenvalue, clamped at zero as the
// reference does (math.rs:34-37).
WMD_HD double msd_from(double gx, double gy, double lambda, double n) {
  const double msd = (gx + gy - 2.0 * lambda) / n;
  return msd > 0.0 ? msd : 0.0;
}

// Rotation mapping frame coordinates onto the reference: R = V U^T with the
// reflection fix, from the SVD.  Used when the eigenvector is ill-defined.
WMD_HD void rotation_from_svd(const double h[9], double r[9]) {
  double s[3], u[9], v[9];
  svd3_jacobi(h, s, u, v);
  // order columns by singular value, descending
  int o0 = 0, o1 = 1, o2 = 2, t;
  if (s[o1] > s[o0]) { t = o0; o0 = o1; o1 = t; }
  if (s[o2] > s[o1]) { t = o1; o1 = o2; o2 = t; }
  if (s[o1] > s[o0]) { t = o0; o0 = o1; o1 = t; }
  const int ord[3] = {o0, o1, o2};
  double uu[9], vs[9];
  for (int j = 0; j < 3; ++j)
    for (int rr = 0; rr < 3; ++rr) {
      uu[rr * 3 + j] = u[rr * 3 + ord[j]];
      vs[rr * 3 + j] = v[rr * 3 + ord[j]];
    }
  // complete U where singular values vanish
  const double smax = s[o0];
  const bool have1 = s[o1] > 1e-15 * smax && s[o1] > 0;
  const bool have2 = s[o2] > 1e-15 * smax && s[o2] > 0;
  if (!(smax > 0)) {
    for (int i = 0; i < 9; ++i) r[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  if (!have1) {
    const double x = uu[0], y = uu[3], z = uu[6];
    double px, py, pz;
    if (fabs(x) < 0.9) { px = 0; py = -z; pz = y; } else { px = -y; py = x; pz = 0; }
    const double nn = sqrt(px * px + py * py + pz * pz);
    uu[1] = px / nn; uu[4] = py / nn; uu[7] = pz / nn;
  }
  if (!have2 || !have1) {
    uu[2] = uu[3] * uu[7] - uu[6] * uu[4];
    uu[5] = uu[6] * uu[1] - uu[0] * uu[7];
    uu[8] = uu[0] * uu[4] - uu[3] * uu[1];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int kk = 0; kk < 3; ++kk) acc += vs[i * 3 + kk] * uu[j * 3 + kk];
      r[i * 3 + j] = acc;
    }
  if (det3(r) < 0.0) {
    for (int i = 0; i < 3; ++i) vs[i * 3 + 2] = -vs[i * 3 + 2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double acc = 0;
        for (int kk = 0; kk < 3; ++kk) acc += vs[i * 3 + kk] * uu[j * 3 + kk];
        r[i * 3 + j] = acc;
      }
  }
}

// Rotation from the QCP eigenvector of K(H) for eigenvalue lambda: the
// eigenvector is a column of adj(K - lambda I); the column with the largest
// diagonal entry is the best conditioned.  Falls back to the SVD rotation when
// the adjugate vanishes (degenerate lambda_max).  The adjugate comes from the
// Laplace expansion over the 2x2 minors of rows {0,1} and {2,3}, written out
// entry by entry so that everything stays in registers.
WMD_HD void rotation_from_qcp(const double h[9], double lambda, double r[9]) {
  double k[16];
  key_matrix(h, k);
  k[0] -= lambda; k[5] -= lambda; k[10] -= lambda; k[15] -= lambda;
  // 2x2 minors of the top rows (s) and bottom rows (c), column pairs
  // (01, 02, 03, 12, 13, 23)
  const double s01 = k[0] * k[5] - k[4] * k[1], s02 = k[0] * k[6] - k[4] * k[2], s03 = k[0] * k[7] - k[4] * k[3];
  const double s12 = k[1] * k[6] - k[5] * k[2], s13 = k[1] * k[7] - k[5] * k[3], s23 = k[2] * k[7] - k[6] * k[3];
  const double c01 = k[8] * k[13] - k[12] * k[9], c02 = k[8] * k[14] - k[12] * k[10];
  const double c03 = k[8] * k[15] - k[12] * k[11], c12 = k[9] * k[14] - k[13] * k[10];
  const double c13 = k[9] * k[15] - k[13] * k[11], c23 = k[10] * k[15] - k[14] * k[11];
  // adjugate a[i][j] = cofactor C_ji
  const double a00 = k[5] * c23 - k[6] * c13 + k[7] * c12;
  const double a01 = -k[1] * c23 + k[2] * c13 - k[3] * c12;
  const double a02 = k[13] * s23 - k[14] * s13 + k[15] * s12;
  const double a03 = -k[9] * s23 + k[10] * s13 - k[11] * s12;
  const double a10 = -k[4] * c23 + k[6] * c03 - k[7] * c02;
  const double a11 = k[0] * c23 - k[2] * c03 + k[3] * c02;
  const double a12 = -k[12] * s23 + k[14] * s03 - k[15] * s02;
  const double a13 = k[8] * s23 - k[10] * s03 + k[11] * s02;
  const double a20 = k[4] * c13 - k[5] * c03 + k[7] * c01;
  const double a21 = -k[0] * c13 + k[1] * c03 - k[3] * c01;
  const double a22 = k[12] * s13 - k[13] * s03 + k[15] * s01;
  const double a23 = -k[8] * s13 + k[9] * s03 - k[11] * s01;
  const double a30 = -k[4] * c12 + k[5] * c02 - k[6] * c01;
  const double a31 = k[0] * c12 - k[1] * c02 + k[2] * c01;
  const double a32 = -k[12] * s12 + k[13] * s02 - k[14] * s01;
  const double a33 = k[8] * s12 - k[9] * s02 + k[10] * s01;
  // column m of the adjugate, m = argmax |a_mm|
  int m = 0;
  double best = fabs(a00);
  if (fabs(a11) > best) { best = fabs(a11); m = 1; }
  if (fabs(a22) > best) { best = fabs(a22); m = 2; }
  if (fabs(a33) > best) { best = fabs(a33); m = 3; }
  double q[4];
  q[0] = m == 0 ? a00 : m == 1 ? a01 : m == 2 ? a02 : a03;
  q[1] = m == 0 ? a10 : m == 1 ? a11 : m == 2 ? a12 : a13;
  q[2] = m == 0 ? a20 : m == 1 ? a21 : m == 2 ? a22 : a23;
  q[3] = m == 0 ? a30 : m == 1 ? a31 : m == 2 ? a32 : a33;
  const double norm2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  // scale-free degeneracy test: |adj column|^2 vs (|K|_F^3)^2
  double kf = 0.0;
  for (int i = 0; i < 16; ++i) kf += k[i] * k[i];
  if (!(norm2 > 1e-24 * kf * kf * kf)) {
    rotation_from_svd(h, r);
    return;
  }
  const double inv = 1.0 / sqrt(norm2);
  const double w = q[0] * inv, x = q[1] * inv, y = q[2] * inv, z = q[3] * inv;
  r[0] = w * w + x * x - y * y - z * z;
  r[1] = 2.0 * (x * y - w * z);
  r[2] = 2.0 * (x * z + w * y);
  r[3] = 2.0 * (x * y + w * z);
  r[4] = w * w - x * x + y * y - z * z;
  r[5] = 2.0 * (y * z - w * x);
  r[6] = 2.0 * (x * z - w * y);
  r[7] = 2.0 * (y * z + w * x);
  r[8] = w * w - x * x - y * y + z * z;
}

}  // namespace wmd

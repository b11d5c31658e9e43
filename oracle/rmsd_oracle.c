/*
 * rmsd_oracle.c -- CPU FP64 restatement of warp-md's RMSD plans.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * warp-md_b200/: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py load it.  Nothing in the product links it.
 *
 * What it restates (reference = warp-md 0.4.30, Rust):
 *   - rmsd_aligned_selected   crates/traj-engine/src/plans/rmsd/plan.rs:1161-1248
 *       two-pass FP64 centroid + covariance H = sum (x-cx)(y-cy)^T, 3x3 SVD,
 *       R = V U^T with the reflection fix (negate the last row of V^T when
 *       det R < 0), explicit residual pass, result rounded to f32.
 *   - rmsd_raw_selected       plan.rs:1093-1110   (align = false)
 *   - rmsd_aligned            plan.rs:1112-1159   (pairwise metric "rms")
 *   - rmsd_raw                plan.rs:1081-1091   (pairwise metric "nofit")
 *   - PairwiseRmsdPlan::finalize  plan.rs:593-674 (symmetric fill, zero
 *       diagonal, n_sel < 2 -> all zeros); metric "dme" plan.rs:612-645 with
 *       pair_distances_compact plan.rs:1279-1302 and apply_pbc
 *       (crates/traj-core/src/pbc_math.rs:17-27)
 *   - AlignPlan / SuperposePlan   crates/traj-engine/src/plans/geometry/align/
 *       plan_exec.rs:125-266, 325-459 with kabsch_rotation_weighted and
 *       centroid_weighted (crates/traj-engine/src/plans/geometry/
 *       geometry_math.rs:202-300): weighted Kabsch, t = cy - R cx, R x + t.
 *   - RmsfPlan / AtomicAdpPlan / RmsdPerResPlan
 *       crates/traj-engine/src/plans/geometry/rms.rs:110-218, 345-429, 633-671.
 *   - TrajectoryClusterPlan (DBSCAN, k-means)
 *       crates/traj-engine/src/plans/analysis/clustering.rs:269-548.
 *
 * The SVD in the reference is nalgebra 0.32.6 (Cargo.lock:792-793), which is
 * not vendored.  Here it is a one-sided Jacobi SVD (Hestenes 1958; Demmel &
 * Veselic 1992) with singular values sorted in descending order, which is the
 * ordering the reference's reflection fix relies on.  Any correct SVD yields
 * the same minimum RMSD.
 *
 * Also here, for cross-checks: the QCP characteristic-polynomial route
 * (Theobald 2005, Acta Cryst A61:478; Liu, Agrafiotis & Theobald 2010) and the
 * analytic gradient dRMSD/dx_k = (x_k - cx - R^T (y_k - cy)) / (n RMSD).
 * The reference has no gradient; this one is checked by central differences.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define WMDO_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* 3x3 helpers (row-major)                                             */
/* ------------------------------------------------------------------ */
static double det3(const double m[9]) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

/* One-sided Jacobi SVD of a 3x3 matrix A = U diag(s) V^T, s sorted
 * descending, U and V orthogonal (U completed by cross products when A is
 * rank deficient).  Returns 0. */
WMDO_API int wmdo_svd3(const double a_in[9], double u[9], double s[3], double vt[9]) {
  double a[9], v[9];
  memcpy(a, a_in, sizeof(a));
  for (int i = 0; i < 9; ++i) v[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    int rotated = 0;
    for (int p = 0; p < 2; ++p) {
      for (int q = p + 1; q < 3; ++q) {
        double alpha = 0, beta = 0, gamma = 0;
        for (int k = 0; k < 3; ++k) {
          alpha += a[k * 3 + p] * a[k * 3 + p];
          beta += a[k * 3 + q] * a[k * 3 + q];
          gamma += a[k * 3 + p] * a[k * 3 + q];
        }
        if (gamma == 0.0 || fabs(gamma) <= 1e-17 * sqrt(alpha * beta)) continue;
        rotated = 1;
        double zeta = (beta - alpha) / (2.0 * gamma);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
        for (int k = 0; k < 3; ++k) {
          double ap = a[k * 3 + p], aq = a[k * 3 + q];
          a[k * 3 + p] = c * ap - sn * aq;
          a[k * 3 + q] = sn * ap + c * aq;
          double vp = v[k * 3 + p], vq = v[k * 3 + q];
          v[k * 3 + p] = c * vp - sn * vq;
          v[k * 3 + q] = sn * vp + c * vq;
        }
      }
    }
    if (!rotated) break;
  }
  double sv[3];
  int order[3] = {0, 1, 2};
  for (int j = 0; j < 3; ++j)
    sv[j] = sqrt(a[0 * 3 + j] * a[0 * 3 + j] + a[1 * 3 + j] * a[1 * 3 + j] + a[2 * 3 + j] * a[2 * 3 + j]);
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (sv[order[j]] > sv[order[i]]) { int t = order[i]; order[i] = order[j]; order[j] = t; }
  double uu[9];
  double smax = sv[order[0]];
  int have[3] = {0, 0, 0};
  for (int jj = 0; jj < 3; ++jj) {
    int j = order[jj];
    s[jj] = sv[j];
    for (int k = 0; k < 3; ++k) vt[jj * 3 + k] = v[k * 3 + j];
    if (sv[j] > 1e-300 && sv[j] > smax * 1e-15) {
      for (int k = 0; k < 3; ++k) uu[k * 3 + jj] = a[k * 3 + j] / sv[j];
      have[jj] = 1;
    }
  }
  /* complete U for rank-deficient inputs */
  if (!have[0]) { uu[0] = 1; uu[3] = 0; uu[6] = 0; have[0] = 1; }
  if (!have[1]) {
    /* any unit vector orthogonal to u0 */
    double x = uu[0], y = uu[3], z = uu[6];
    double px, py, pz;
    if (fabs(x) < 0.9) { px = 0; py = -z; pz = y; } else { px = -y; py = x; pz = 0; }
    double nn = sqrt(px * px + py * py + pz * pz);
    uu[1] = px / nn; uu[4] = py / nn; uu[7] = pz / nn;
    have[1] = 1;
  }
  if (!have[2]) {
    uu[2] = uu[3] * uu[7] - uu[6] * uu[4];
    uu[5] = uu[6] * uu[1] - uu[0] * uu[7];
    uu[8] = uu[0] * uu[4] - uu[3] * uu[1];
  }
  memcpy(u, uu, sizeof(uu));
  return 0;
}

/* R = V U^T with the reference's reflection fix. */
static void kabsch_rotation(const double h[9], double r[9], double* sigma_sum) {
  double u[9], s[3], vt[9];
  wmdo_svd3(h, u, s, vt);
  /* r = vt^T * u^T  -> r[i][j] = sum_k vt[k][i] * u[j][k] */
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += vt[k * 3 + i] * u[j * 3 + k];
      r[i * 3 + j] = acc;
    }
  double ss = s[0] + s[1] + s[2];
  if (det3(r) < 0.0) {
    for (int k = 0; k < 3; ++k) vt[2 * 3 + k] = -vt[2 * 3 + k];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double acc = 0;
        for (int k = 0; k < 3; ++k) acc += vt[k * 3 + i] * u[j * 3 + k];
        r[i * 3 + j] = acc;
      }
    ss -= 2.0 * s[2];
  }
  if (sigma_sum) *sigma_sum = ss;
}

/* ------------------------------------------------------------------ */
/* Per-frame plans                                                     */
/* ------------------------------------------------------------------ */

/* plan.rs:1093-1110 */
static double raw_selected(const float* frame, int64_t frame_atoms, int stride, const float* ref,
                           int ref_stride, const uint32_t* sel, int64_t n) {
  if (n == 0) return 0.0;
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    int64_t idx = sel ? (int64_t)sel[i] : i;
    if (idx >= frame_atoms) break;
    const float* p = frame + idx * stride;
    const float* q = ref + i * ref_stride;
    double dx = (double)p[0] - (double)q[0];
    double dy = (double)p[1] - (double)q[1];
    double dz = (double)p[2] - (double)q[2];
    sum += dx * dx + dy * dy + dz * dz;
  }
  return sqrt(sum / (double)n);
}

/* plan.rs:1161-1248.  Returns RMSD in FP64 (the reference rounds it to f32);
 * optionally returns the rotation, centroids (for the gradient). */
static double aligned_selected(const float* frame, int64_t frame_atoms, int stride, const float* ref,
                               int ref_stride, const uint32_t* sel, int64_t n, double r_out[9],
                               double cx_out[3], double cy_out[3]) {
  if (n == 0) return 0.0;
  double cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i) {
    int64_t idx = sel ? (int64_t)sel[i] : i;
    if (idx >= frame_atoms) return 0.0;
    const float* p = frame + idx * stride;
    const float* q = ref + i * ref_stride;
    cx[0] += p[0]; cx[1] += p[1]; cx[2] += p[2];
    cy[0] += q[0]; cy[1] += q[1]; cy[2] += q[2];
  }
  double inv_n = 1.0 / (double)n;
  for (int k = 0; k < 3; ++k) { cx[k] *= inv_n; cy[k] *= inv_n; }
  double h[9] = {0};
  for (int64_t i = 0; i < n; ++i) {
    int64_t idx = sel ? (int64_t)sel[i] : i;
    const float* p = frame + idx * stride;
    const float* q = ref + i * ref_stride;
    double px = p[0] - cx[0], py = p[1] - cx[1], pz = p[2] - cx[2];
    double qx = q[0] - cy[0], qy = q[1] - cy[1], qz = q[2] - cy[2];
    h[0] += px * qx; h[1] += px * qy; h[2] += px * qz;
    h[3] += py * qx; h[4] += py * qy; h[5] += py * qz;
    h[6] += pz * qx; h[7] += pz * qy; h[8] += pz * qz;
  }
  double r[9];
  kabsch_rotation(h, r, NULL);
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    int64_t idx = sel ? (int64_t)sel[i] : i;
    const float* p = frame + idx * stride;
    const float* q = ref + i * ref_stride;
    double px = p[0] - cx[0], py = p[1] - cx[1], pz = p[2] - cx[2];
    double qx = q[0] - cy[0], qy = q[1] - cy[1], qz = q[2] - cy[2];
    double ax = r[0] * px + r[1] * py + r[2] * pz;
    double ay = r[3] * px + r[4] * py + r[5] * pz;
    double az = r[6] * px + r[7] * py + r[8] * pz;
    double dx = ax - qx, dy = ay - qy, dz = az - qz;
    sum += dx * dx + dy * dy + dz * dz;
  }
  if (r_out) memcpy(r_out, r, sizeof(r));
  if (cx_out) memcpy(cx_out, cx, sizeof(cx));
  if (cy_out) memcpy(cy_out, cy, sizeof(cy));
  return sqrt(sum * inv_n);
}

/* RmsdPlan over a frame-major trajectory: coords [n_frames][n_atoms][stride],
 * reference [n_sel][ref_stride] (already the selected atoms, as the plan
 * stores it), sel = NULL means the dense selection 0..n_sel-1.
 * out32 receives the reference's f32 result, out64 (nullable) the FP64 value
 * before rounding.  n_threads <= 0 means all OpenMP threads. */
WMDO_API void wmdo_rmsd_frames(const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                               const uint32_t* sel, int64_t n_sel, const float* ref, int ref_stride,
                               int align, float* out32, double* out64, int n_threads) {
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
  for (int64_t f = 0; f < n_frames; ++f) {
    const float* frame = coords + f * n_atoms * stride;
    double v = align ? aligned_selected(frame, n_atoms, stride, ref, ref_stride, sel, n_sel, NULL, NULL, NULL)
                     : raw_selected(frame, n_atoms, stride, ref, ref_stride, sel, n_sel);
    if (out32) out32[f] = (float)v;
    if (out64) out64[f] = v;
  }
  (void)n_threads;
}

/* Analytic FP64 gradient of the aligned RMSD w.r.t. the frame coordinates:
 * grad[f][i][:] = (x_i - cx - R^T (y_i - cy)) / (n * rmsd), zero when rmsd == 0.
 * Writes only the selected atoms' rows (grad has the layout of coords with
 * stride 3; unselected atoms are left untouched). */
WMDO_API void wmdo_rmsd_grad(const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                             const uint32_t* sel, int64_t n_sel, const float* ref, int ref_stride,
                             double* rmsd_out, double* grad, int n_threads) {
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
  for (int64_t f = 0; f < n_frames; ++f) {
    const float* frame = coords + f * n_atoms * stride;
    double r[9], cx[3], cy[3];
    double v = aligned_selected(frame, n_atoms, stride, ref, ref_stride, sel, n_sel, r, cx, cy);
    if (rmsd_out) rmsd_out[f] = v;
    double scale = (v > 0.0 && n_sel > 0) ? 1.0 / ((double)n_sel * v) : 0.0;
    for (int64_t i = 0; i < n_sel; ++i) {
      int64_t idx = sel ? (int64_t)sel[i] : i;
      const float* p = frame + idx * stride;
      const float* q = ref + i * ref_stride;
      double qx = q[0] - cy[0], qy = q[1] - cy[1], qz = q[2] - cy[2];
      /* R^T q */
      double tx = r[0] * qx + r[3] * qy + r[6] * qz;
      double ty = r[1] * qx + r[4] * qy + r[7] * qz;
      double tz = r[2] * qx + r[5] * qy + r[8] * qz;
      double* g = grad + (f * n_atoms + idx) * 3;
      g[0] = (p[0] - cx[0] - tx) * scale;
      g[1] = (p[1] - cx[1] - ty) * scale;
      g[2] = (p[2] - cx[2] - tz) * scale;
    }
  }
  (void)n_threads;
}

/* ------------------------------------------------------------------ */
/* Pairwise plan (plan.rs:593-674 with rmsd_aligned / rmsd_raw)        */
/* ------------------------------------------------------------------ */

/* plan.rs:1112-1159: frame = frames[i], reference = frames[j] */
static double pair_aligned(const float* a, const float* b, int64_t n, int stride) {
  return aligned_selected(a, n, stride, b, stride, NULL, n, NULL, NULL, NULL);
}

/* plan.rs:1081-1091 */
static double pair_raw(const float* a, const float* b, int64_t n, int stride) {
  return raw_selected(a, n, stride, b, stride, NULL, n);
}

/* Fills rows [i0,i1) x cols [j0,j1) of the pairwise matrix of the frames in
 * `frames` ([n_frames][n_sel][stride], already selected).  metric 0 = rms,
 * 1 = nofit.  out32 (and optional out64) are row-major with leading dimension
 * ld.  The diagonal is 0; n_sel < 2 gives zeros (plan.rs:604-610). */
WMDO_API void wmdo_pairwise_block(const float* frames, int64_t n_frames, int64_t n_sel, int stride,
                                  int metric, int64_t i0, int64_t i1, int64_t j0, int64_t j1,
                                  float* out32, double* out64, int64_t ld, int n_threads) {
  (void)n_frames;
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
  for (int64_t i = i0; i < i1; ++i) {
    for (int64_t j = j0; j < j1; ++j) {
      double v = 0.0;
      if (i != j && n_sel >= 2) {
        /* the reference computes pair (min, max) and mirrors it */
        int64_t a = i < j ? i : j, b = i < j ? j : i;
        const float* fa = frames + a * n_sel * stride;
        const float* fb = frames + b * n_sel * stride;
        v = metric == 0 ? pair_aligned(fa, fb, n_sel, stride) : pair_raw(fa, fb, n_sel, stride);
      }
      if (out32) out32[(i - i0) * ld + (j - j0)] = (float)v;
      if (out64) out64[(i - i0) * ld + (j - j0)] = v;
    }
  }
  (void)n_threads;
}

/* ------------------------------------------------------------------ */
/* Pairwise metric "dme" (distance-matrix error)                        */
/* ------------------------------------------------------------------ */

/* pair_distances_compact (plan.rs:1279-1302) with apply_pbc
 * (crates/traj-core/src/pbc_math.rs:17-27): every atom pair a < b in
 * lexicographic order, the coordinate difference taken in f32 and widened to
 * f64; with a box, the minimum image per axis whose length is > 0
 * (d -= round(d / L) * L, round half away from zero); distance in f64. */
static void dme_distances(const float* frame, int64_t n, int stride, const float* box, double* out) {
  const double lx = box ? (double)box[0] : 0.0, ly = box ? (double)box[1] : 0.0, lz = box ? (double)box[2] : 0.0;
  int64_t k = 0;
  for (int64_t a = 0; a < n; ++a) {
    const float* pa = frame + a * stride;
    for (int64_t b = a + 1; b < n; ++b) {
      const float* pb = frame + b * stride;
      double dx = (double)(float)(pb[0] - pa[0]);
      double dy = (double)(float)(pb[1] - pa[1]);
      double dz = (double)(float)(pb[2] - pa[2]);
      if (box) {
        if (lx > 0.0) dx -= round(dx / lx) * lx;
        if (ly > 0.0) dy -= round(dy / ly) * ly;
        if (lz > 0.0) dz -= round(dz / lz) * lz;
      }
      out[k++] = sqrt(dx * dx + dy * dy + dz * dz);
    }
  }
}

/* PairwiseRmsdPlan::finalize for metric Dme (plan.rs:612-645): per frame pair
 * i < j, sqrt(sum_k (d_i[k] - d_j[k])^2 / n_pairs), the sum in pair order, the
 * result rounded to f32 and mirrored; zero diagonal; n_sel < 2 -> zeros.
 * frames: already-selected atoms [n_frames][n_sel][stride]; box: per-frame
 * orthorhombic lengths [n_frames][3] (pbc "orthorhombic") or NULL ("none"). */
WMDO_API void wmdo_pairwise_dme(const float* frames, int64_t n_frames, int64_t n_sel, int stride, const float* box,
                                float* out32, double* out64, int n_threads) {
  const int64_t nn = n_frames * n_frames;
  for (int64_t e = 0; e < nn; ++e) {
    if (out32) out32[e] = 0.f;
    if (out64) out64[e] = 0.0;
  }
  if (n_sel < 2 || n_frames == 0) return;
  const int64_t n_pairs = n_sel * (n_sel - 1) / 2;
  double* d = (double*)malloc((size_t)n_frames * (size_t)n_pairs * sizeof(double));
  if (!d) return;
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
  for (int64_t f = 0; f < n_frames; ++f)
    dme_distances(frames + f * n_sel * stride, n_sel, stride, box ? box + f * 3 : NULL, d + f * n_pairs);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
  for (int64_t i = 0; i < n_frames; ++i) {
    for (int64_t j = i + 1; j < n_frames; ++j) {
      const double* di = d + i * n_pairs;
      const double* dj = d + j * n_pairs;
      double sum = 0.0;
      for (int64_t k = 0; k < n_pairs; ++k) {
        const double diff = di[k] - dj[k];
        sum += diff * diff;
      }
      const double v = sqrt(sum / (double)n_pairs);
      if (out32) out32[i * n_frames + j] = out32[j * n_frames + i] = (float)v;
      if (out64) out64[i * n_frames + j] = out64[j * n_frames + i] = v;
    }
  }
  free(d);
  (void)n_threads;
}

/* ------------------------------------------------------------------ */
/* QCP cross-check (Theobald 2005)                                     */
/* ------------------------------------------------------------------ */

static double det4(const double k[16]) {
  double s0 = k[0] * k[5] - k[1] * k[4];
  double s1 = k[0] * k[6] - k[2] * k[4];
  double s2 = k[0] * k[7] - k[3] * k[4];
  double s3 = k[1] * k[6] - k[2] * k[5];
  double s4 = k[1] * k[7] - k[3] * k[5];
  double s5 = k[2] * k[7] - k[3] * k[6];
  double c5 = k[10] * k[15] - k[11] * k[14];
  double c4 = k[9] * k[15] - k[11] * k[13];
  double c3 = k[9] * k[14] - k[10] * k[13];
  double c2 = k[8] * k[15] - k[11] * k[12];
  double c1 = k[8] * k[14] - k[10] * k[12];
  double c0 = k[8] * k[13] - k[9] * k[12];
  return s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
}

/* RMSD of one frame against one reference by QCP in FP64 (centroids and
 * G terms computed two-pass in FP64).  Long-double Newton when hp != 0. */
WMDO_API double wmdo_qcp_rmsd(const float* x, const float* y, int64_t n, int stride, int hp) {
  if (n == 0) return 0.0;
  double cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) { cx[k] += x[i * stride + k]; cy[k] += y[i * stride + k]; }
  for (int k = 0; k < 3; ++k) { cx[k] /= (double)n; cy[k] /= (double)n; }
  double h[9] = {0}, gx = 0, gy = 0;
  for (int64_t i = 0; i < n; ++i) {
    double p[3], q[3];
    for (int k = 0; k < 3; ++k) { p[k] = x[i * stride + k] - cx[k]; q[k] = y[i * stride + k] - cy[k]; }
    for (int a = 0; a < 3; ++a) {
      gx += p[a] * p[a];
      gy += q[a] * q[a];
      for (int b = 0; b < 3; ++b) h[a * 3 + b] += p[a] * q[b];
    }
  }
  double sxx = h[0], sxy = h[1], sxz = h[2], syx = h[3], syy = h[4], syz = h[5], szx = h[6], szy = h[7], szz = h[8];
  double K[16] = {sxx + syy + szz, syz - szy, szx - sxz, sxy - syx,
                  syz - szy, sxx - syy - szz, sxy + syx, szx + sxz,
                  szx - sxz, sxy + syx, -sxx + syy - szz, syz + szy,
                  sxy - syx, szx + sxz, syz + szy, -sxx - syy + szz};
  double c2 = 0;
  for (int i = 0; i < 9; ++i) c2 += h[i] * h[i];
  c2 *= -2.0;
  double c1 = -8.0 * det3(h);
  double c0 = det4(K);
  double e0 = 0.5 * (gx + gy);
  double lambda;
  if (hp) {
    long double l = e0;
    for (int it = 0; it < 200; ++it) {
      long double l2 = l * l;
      long double p = l2 * l2 + c2 * l2 + c1 * l + c0;
      long double dp = 4 * l2 * l + 2 * c2 * l + c1;
      if (dp == 0) break;
      long double nl = l - p / dp;
      if (fabsl(nl - l) <= 1e-19L * fabsl(nl)) { l = nl; break; }
      l = nl;
    }
    lambda = (double)l;
  } else {
    double l = e0;
    for (int it = 0; it < 200; ++it) {
      double l2 = l * l;
      double p = l2 * l2 + c2 * l2 + c1 * l + c0;
      double dp = 4 * l2 * l + 2 * c2 * l + c1;
      if (dp == 0) break;
      double nl = l - p / dp;
      if (fabs(nl - l) <= 1e-15 * fabs(nl)) { l = nl; break; }
      l = nl;
    }
    lambda = l;
  }
  double msd = (gx + gy - 2.0 * lambda) / (double)n;
  return msd > 0 ? sqrt(msd) : 0.0;
}

/* Kabsch rotation for an arbitrary covariance (exposed for tests of the
 * rotation convention): r maps frame coordinates onto the reference. */
WMDO_API void wmdo_kabsch_rotation(const double h[9], double r[9], double* sigma_sum) {
  kabsch_rotation(h, r, sigma_sum);
}

/* ------------------------------------------------------------------ */
/* Superposition plans (AlignPlan / SuperposePlan)                     */
/* ------------------------------------------------------------------ */

/* centroid_weighted (crates/traj-engine/src/plans/geometry/geometry_math.rs:
 * 202-233): weighted mean, 0 when the weights sum to 0. */
static void centroid_w(const float* pts, int stride, const uint32_t* sel, int64_t n, const float* w, double c[3]) {
  double s[3] = {0, 0, 0}, ws = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t idx = sel ? (int64_t)sel[i] : i;
    const float* p = pts + idx * stride;
    const double wi = w ? (double)w[i] : 1.0;
    s[0] += (double)p[0] * wi; s[1] += (double)p[1] * wi; s[2] += (double)p[2] * wi;
    ws += wi;
  }
  if (!w) ws = (double)n;
  for (int k = 0; k < 3; ++k) c[k] = ws == 0.0 ? 0.0 : s[k] / ws;
}

/* Per frame: kabsch_rotation_weighted (geometry_math.rs:235-300) of the
 * selection onto the reference -- weighted centroids, H = sum w (x - cx)
 * (y - cy)^T, R = V U^T with the reflection fix; norotate: R = I -- then
 * t = cy - R cx (plan_exec.rs:224 / 415).  xf [n_frames][12] = R row-major,
 * t.  When out is not NULL every atom of the frame is moved: out = R x + t in
 * FP64, rounded to f32 (plan_exec.rs:431-444). */
WMDO_API void wmdo_superpose(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                             int64_t n_sel, const float* ref, int ref_stride, const float* weights, int norotate,
                             double* xf, float* out, int n_threads) {
#ifdef _OPENMP
  int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
  for (int64_t f = 0; f < n_frames; ++f) {
    const float* frame = coords + f * n_atoms * stride;
    double r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
    if (n_sel > 0) {
      centroid_w(frame, stride, sel, n_sel, weights, cx);
      centroid_w(ref, ref_stride, NULL, n_sel, weights, cy);
      if (!norotate) {
        double h[9] = {0};
        for (int64_t i = 0; i < n_sel; ++i) {
          const int64_t idx = sel ? (int64_t)sel[i] : i;
          const float* p = frame + idx * stride;
          const float* q = ref + i * ref_stride;
          const double wi = weights ? (double)weights[i] : 1.0;
          const double px = p[0] - cx[0], py = p[1] - cx[1], pz = p[2] - cx[2];
          const double qx = q[0] - cy[0], qy = q[1] - cy[1], qz = q[2] - cy[2];
          h[0] += px * qx * wi; h[1] += px * qy * wi; h[2] += px * qz * wi;
          h[3] += py * qx * wi; h[4] += py * qy * wi; h[5] += py * qz * wi;
          h[6] += pz * qx * wi; h[7] += pz * qy * wi; h[8] += pz * qz * wi;
        }
        kabsch_rotation(h, r, NULL);
      }
    }
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = cy[i] - (r[i * 3] * cx[0] + r[i * 3 + 1] * cx[1] + r[i * 3 + 2] * cx[2]);
    if (xf) {
      memcpy(xf + f * 12, r, sizeof(r));
      memcpy(xf + f * 12 + 9, t, sizeof(t));
    }
    if (out) {
      float* o = out + f * n_atoms * 3;
      for (int64_t a = 0; a < n_atoms; ++a) {
        const float* p = frame + a * stride;
        const double x = p[0], y = p[1], z = p[2];
        o[a * 3 + 0] = (float)(r[0] * x + r[1] * y + r[2] * z + t[0]);
        o[a * 3 + 1] = (float)(r[3] * x + r[4] * y + r[5] * z + t[1]);
        o[a * 3 + 2] = (float)(r[6] * x + r[7] * y + r[8] * z + t[2]);
      }
    }
  }
  (void)n_threads;
}

/* ------------------------------------------------------------------ */
/* Fluctuations and per-residue RMSD                                   */
/* ------------------------------------------------------------------ */

/* RmsfPlan CPU path (crates/traj-engine/src/plans/geometry/rms.rs:110-140,
 * 193-218): Welford running mean / M2 per selected atom and axis, FP64;
 * rmsf = sqrt((M2x + M2y + M2z) / n).  AtomicAdpPlan (rms.rs:345-429): raw
 * sums of x and of the six products, u_ab = <ab> - <a><b>, diagonal clamped
 * at 0.  Either output may be NULL. */
WMDO_API void wmdo_rmsf(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                        int64_t n_sel, double* rmsf, double* adp) {
  for (int64_t i = 0; i < n_sel; ++i) {
    const int64_t a = sel ? (int64_t)sel[i] : i;
    double mean[3] = {0, 0, 0}, m2[3] = {0, 0, 0}, s[3] = {0, 0, 0}, pr[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t f = 0; f < n_frames; ++f) {
      const float* p = coords + (f * n_atoms + a) * stride;
      const double n = (double)(f + 1);
      for (int c = 0; c < 3; ++c) {
        const double x = p[c];
        const double d = x - mean[c];
        mean[c] += d / n;
        m2[c] += d * (x - mean[c]);
        s[c] += x;
      }
      const double x = p[0], y = p[1], z = p[2];
      pr[0] += x * x; pr[1] += y * y; pr[2] += z * z; pr[3] += x * y; pr[4] += x * z; pr[5] += y * z;
    }
    if (rmsf) rmsf[i] = n_frames ? sqrt((m2[0] + m2[1] + m2[2]) / (double)n_frames) : 0.0;
    if (adp && n_frames) {
      const double inv = 1.0 / (double)n_frames;
      const double mx = s[0] * inv, my = s[1] * inv, mz = s[2] * inv;
      double* o = adp + i * 6;
      o[0] = fmax(pr[0] * inv - mx * mx, 0.0);
      o[1] = fmax(pr[1] * inv - my * my, 0.0);
      o[2] = fmax(pr[2] * inv - mz * mz, 0.0);
      o[3] = pr[3] * inv - mx * my;
      o[4] = pr[4] * inv - mx * mz;
      o[5] = pr[5] * inv - my * mz;
    }
  }
}

/* RmsdPerResPlan CPU path (rms.rs:633-671): per frame the unweighted Kabsch of
 * the selection onto ref_all[sel] (kabsch_rotation), then per group
 * sqrt(sum |R (x - cx) - (y - cy)|^2 / max(n, 1)); align = 0 compares raw
 * coordinates.  out [n_frames][n_groups] in FP64 (the reference rounds to f32). */
WMDO_API void wmdo_rmsd_perres(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                               int64_t n_sel, const float* ref_all, const uint32_t* goff, const uint32_t* gatoms,
                               int64_t n_groups, int align, double* out) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4)
#endif
  for (int64_t f = 0; f < n_frames; ++f) {
    const float* frame = coords + f * n_atoms * stride;
    double r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
    if (align && n_sel > 0) {
      for (int64_t i = 0; i < n_sel; ++i) {
        const int64_t a = sel ? (int64_t)sel[i] : i;
        for (int c = 0; c < 3; ++c) { cx[c] += frame[a * stride + c]; cy[c] += ref_all[a * 3 + c]; }
      }
      for (int c = 0; c < 3; ++c) { cx[c] /= (double)n_sel; cy[c] /= (double)n_sel; }
      double h[9] = {0};
      for (int64_t i = 0; i < n_sel; ++i) {
        const int64_t a = sel ? (int64_t)sel[i] : i;
        double px[3], qy[3];
        for (int c = 0; c < 3; ++c) { px[c] = frame[a * stride + c] - cx[c]; qy[c] = ref_all[a * 3 + c] - cy[c]; }
        for (int u = 0; u < 3; ++u)
          for (int v = 0; v < 3; ++v) h[u * 3 + v] += px[u] * qy[v];
      }
      kabsch_rotation(h, r, NULL);
    }
    for (int64_t g = 0; g < n_groups; ++g) {
      double sum = 0.0;
      for (uint32_t k = goff[g]; k < goff[g + 1]; ++k) {
        const int64_t a = gatoms[k];
        double p[3], q[3];
        for (int c = 0; c < 3; ++c) {
          p[c] = (double)frame[a * stride + c] - (align ? cx[c] : 0.0);
          q[c] = (double)ref_all[a * 3 + c] - (align ? cy[c] : 0.0);
        }
        for (int u = 0; u < 3; ++u) {
          const double d = (align ? r[u * 3] * p[0] + r[u * 3 + 1] * p[1] + r[u * 3 + 2] * p[2] : p[u]) - q[u];
          sum += d * d;
        }
      }
      const double n = goff[g + 1] > goff[g] ? (double)(goff[g + 1] - goff[g]) : 1.0;
      out[f * n_groups + g] = sqrt(sum / n);
    }
  }
}

/* ------------------------------------------------------------------ */
/* Clustering (TrajectoryClusterPlan)                                  */
/* ------------------------------------------------------------------ */

/* dbscan_cluster (crates/traj-engine/src/plans/analysis/clustering.rs:
 * 269-374) over a full n x n float32 distance matrix (tri_get reads the
 * triangle; d(i,i) = 0): sequential DBSCAN with a FIFO queue, then per cluster
 * the member with the smallest FP64 sum of distances (first such index).
 * Returns the number of clusters; centroids/sizes need room for n entries. */
WMDO_API int64_t wmdo_dbscan(const float* D, int64_t n, double eps, int64_t min_samples, int32_t* labels,
                             uint32_t* centroids, uint32_t* sizes) {
  const int32_t UNCLASSIFIED = -2, NOISE = -1;
  if (min_samples < 1) min_samples = 1;
  unsigned char* visited = (unsigned char*)calloc((size_t)n, 1);
  unsigned char* queued = (unsigned char*)malloc((size_t)n);
  int64_t* neigh = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  int64_t* queue = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));  /* each point queued once per cluster */
  for (int64_t i = 0; i < n; ++i) labels[i] = UNCLASSIFIED;
  int32_t cluster = 0;
#define WMDO_D(a, b) ((a) == (b) ? 0.0 : (double)D[(a) * n + (b)])
  for (int64_t i = 0; i < n; ++i) {
    if (visited[i]) continue;
    visited[i] = 1;
    int64_t nn = 0;
    for (int64_t j = 0; j < n; ++j)
      if (WMDO_D(i, j) <= eps) neigh[nn++] = j;
    if (nn < min_samples) {
      labels[i] = NOISE;
      continue;
    }
    labels[i] = cluster;
    memset(queued, 0, (size_t)n);
    int64_t qh = 0, qt = 0;
    for (int64_t k = 0; k < nn; ++k)
      if (neigh[k] != i && !queued[neigh[k]]) {
        queue[qt++] = neigh[k];
        queued[neigh[k]] = 1;
      }
    while (qh < qt) {
      const int64_t p = queue[qh++];
      if (!visited[p]) {
        visited[p] = 1;
        int64_t m = 0;
        for (int64_t j = 0; j < n; ++j)
          if (WMDO_D(p, j) <= eps) neigh[m++] = j;
        if (m >= min_samples)
          for (int64_t k = 0; k < m; ++k)
            if (!queued[neigh[k]]) {
              queue[qt++] = neigh[k];
              queued[neigh[k]] = 1;
            }
      }
      if (labels[p] == UNCLASSIFIED || labels[p] == NOISE) labels[p] = cluster;
    }
    ++cluster;
  }
  for (int32_t c = 0; c < cluster; ++c) {
    uint32_t size = 0, best = 0;
    double best_sum = INFINITY;
    int first = 1;
    for (int64_t a = 0; a < n; ++a) {
      if (labels[a] != c) continue;
      ++size;
      if (first) { best = (uint32_t)a; first = 0; }
      double s = 0.0;
      for (int64_t b = 0; b < n; ++b)
        if (labels[b] == c) s += WMDO_D(a, b);
      if (s < best_sum) { best_sum = s; best = (uint32_t)a; }
    }
    sizes[c] = size;
    centroids[c] = best;
  }
#undef WMDO_D
  free(visited); free(queued); free(neigh); free(queue);
  return cluster;
}

static uint64_t xorshift64_step(uint64_t* state) {
  uint64_t x = *state;
  if (x == 0) x = 0x9E3779B97F4A7C15ull;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *state = x;
  return x;
}

static double sq_dist(const double* a, const double* b, int64_t m) {
  double s = 0.0;
  for (int64_t i = 0; i < m; ++i) {
    const double d = a[i] - b[i];
    s += d * d;
  }
  return s;
}

/* build_aligned_features + kmeans_cluster (clustering.rs:376-548): features
 * are the selection's coordinates after the unweighted Kabsch onto frame 0's,
 * R (x - cx) + cy, in FP64; Lloyd iterations with the xorshift64 shuffle and
 * reseeding.  Returns the number of clusters K. */
WMDO_API int64_t wmdo_kmeans(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                             int64_t n_sel, int64_t n_clusters, int64_t max_iter, double tol, uint64_t seed,
                             int32_t* labels, uint32_t* centroids, uint32_t* sizes) {
  const int64_t N = n_frames, nf = n_sel * 3;
  if (N == 0) return 0;
  int64_t K = n_clusters < 1 ? 1 : (n_clusters > N ? N : n_clusters);
  if (max_iter < 1) max_iter = 1;
  if (tol < 0) tol = 0;
  double* feat = (double*)malloc(sizeof(double) * (size_t)(N * nf));
  const float* ref = coords;  /* frame 0 */
  for (int64_t f = 0; f < N; ++f) {
    const float* fr = coords + f * n_atoms * stride;
    double cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
    for (int64_t i = 0; i < n_sel; ++i) {
      const int64_t a = sel ? (int64_t)sel[i] : i;
      for (int c = 0; c < 3; ++c) { cx[c] += fr[a * stride + c]; cy[c] += ref[a * stride + c]; }
    }
    for (int c = 0; c < 3; ++c) { cx[c] /= (double)n_sel; cy[c] /= (double)n_sel; }
    double h[9] = {0}, r[9];
    for (int64_t i = 0; i < n_sel; ++i) {
      const int64_t a = sel ? (int64_t)sel[i] : i;
      double p[3], q[3];
      for (int c = 0; c < 3; ++c) { p[c] = fr[a * stride + c] - cx[c]; q[c] = ref[a * stride + c] - cy[c]; }
      for (int u = 0; u < 3; ++u)
        for (int v = 0; v < 3; ++v) h[u * 3 + v] += p[u] * q[v];
    }
    kabsch_rotation(h, r, NULL);
    for (int64_t i = 0; i < n_sel; ++i) {
      const int64_t a = sel ? (int64_t)sel[i] : i;
      double p[3];
      for (int c = 0; c < 3; ++c) p[c] = fr[a * stride + c] - cx[c];
      for (int u = 0; u < 3; ++u)
        feat[(f * n_sel + i) * 3 + u] = r[u * 3] * p[0] + r[u * 3 + 1] * p[1] + r[u * 3 + 2] * p[2] + cy[u];
    }
  }
  uint64_t state = seed == 0 ? 0x9E3779B97F4A7C15ull : seed;
  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)N);
  for (int64_t i = 0; i < N; ++i) order[i] = i;
  for (int64_t i = N - 1; i >= 1; --i) {
    const int64_t j = (int64_t)(xorshift64_step(&state) % (uint64_t)(i + 1));
    const int64_t t = order[i]; order[i] = order[j]; order[j] = t;
  }
  double* centers = (double*)malloc(sizeof(double) * (size_t)(K * nf));
  double* sums = (double*)malloc(sizeof(double) * (size_t)(K * nf));
  double* nc = (double*)malloc(sizeof(double) * (size_t)nf);
  int64_t* counts = (int64_t*)malloc(sizeof(int64_t) * (size_t)K);
  for (int64_t c = 0; c < K; ++c) memcpy(centers + c * nf, feat + order[c] * nf, sizeof(double) * (size_t)nf);
  for (int64_t it = 0; it < max_iter; ++it) {
    memset(counts, 0, sizeof(int64_t) * (size_t)K);
    memset(sums, 0, sizeof(double) * (size_t)(K * nf));
    for (int64_t i = 0; i < N; ++i) {
      int64_t best = 0;
      double bd = INFINITY;
      for (int64_t c = 0; c < K; ++c) {
        const double d = sq_dist(feat + i * nf, centers + c * nf, nf);
        if (d < bd) { bd = d; best = c; }
      }
      labels[i] = (int32_t)best;
      counts[best] += 1;
      for (int64_t k = 0; k < nf; ++k) sums[best * nf + k] += feat[i * nf + k];
    }
    double max_shift = 0.0;
    for (int64_t c = 0; c < K; ++c) {
      if (counts[c] == 0) {
        const int64_t idx = (int64_t)(xorshift64_step(&state) % (uint64_t)N);
        const double sh = sqrt(sq_dist(centers + c * nf, feat + idx * nf, nf));
        if (sh > max_shift) max_shift = sh;
        memcpy(centers + c * nf, feat + idx * nf, sizeof(double) * (size_t)nf);
        continue;
      }
      const double inv = 1.0 / (double)counts[c];
      for (int64_t k = 0; k < nf; ++k) nc[k] = sums[c * nf + k] * inv;
      const double sh = sqrt(sq_dist(centers + c * nf, nc, nf));
      if (sh > max_shift) max_shift = sh;
      memcpy(centers + c * nf, nc, sizeof(double) * (size_t)nf);
    }
    if (max_shift <= tol) break;
  }
  for (int64_t c = 0; c < K; ++c) {
    uint32_t cnt = 0, best_idx = 0;
    double bd = INFINITY;
    for (int64_t i = 0; i < N; ++i) {
      if (labels[i] != c) continue;
      ++cnt;
      const double d = sq_dist(feat + i * nf, centers + c * nf, nf);
      if (d < bd) { bd = d; best_idx = (uint32_t)i; }
    }
    sizes[c] = cnt;
    centroids[c] = best_idx;
  }
  free(feat); free(order); free(centers); free(sums); free(nc); free(counts);
  return K;
}

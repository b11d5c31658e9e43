// superpose.cu -- per-frame optimal superposition transforms and their
// application to whole frames (AlignPlan / RotationMatrixPlan /
// SuperposePlan / SuperposeTrajectoryPlan).
//
// The reference computes, per frame on the host, the (optionally
// mass-weighted) Kabsch rotation of the selection onto the reference,
// t = c_y - R c_x, and then R x + t for every atom of the frame
// (crates/traj-engine/src/plans/geometry/align/plan_exec.rs:125-266 and
// 325-459; kabsch_rotation_weighted, geometry_math.rs:235-300).  Here:
//   1. the per-frame statistics stream through rmsd_frames_kernel (weighted
//      mode when the reference carries weights) into tile partials;
//   2. superpose_finalize_kernel sums each frame's partials in tile order and
//      runs, one lane per frame, QCP and the rotation from the QCP
//      eigenvector in FP64 (the same rotation the SVD gives, with the
//      reflection handled by construction), writing the 12-number transform;
//   3. superpose_apply_kernel moves every atom of every frame, FP64
//      arithmetic rounded to float32 as the reference does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_util.cuh"
#include "qcp.cuh"
#include "superpose.h"
#include "wmd_internal.h"

namespace wmd {
namespace {

// One lane per frame.  xf64[f*16 + 0..8] = R (row-major, R (x - c_x) ~ y - c_y),
// [9..11] = t; xf32[f*12 + ...] the same rounded to float32 (optional).
__global__ void __launch_bounds__(256) superpose_finalize_kernel(const FrameLaunch L, int n_tiles, int norotate,
                                                                 double* __restrict__ xf64,
                                                                 float* __restrict__ xf32) {
  __shared__ double st[8][32][17];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = ((int64_t)blockIdx.x * 8 + warp) * 32;
  if (base >= L.n_frames) return;
  for (int i = 0; i < 16; ++i) {
    const int fl = 2 * i + (lane >> 4);
    const int64_t f = base + fl;
    double v = 0.0;
    if (f < L.n_frames) {
      const double* part = L.partial + (size_t)f * n_tiles * kStatDoubles + (lane & 15);
      for (int t = 0; t < n_tiles; ++t) v += part[(size_t)t * kStatDoubles];
    }
    st[warp][fl][lane & 15] = v;
  }
  __syncwarp();
  const int64_t f = base + lane;
  if (f >= L.n_frames) return;
  const double* tot = st[warp][lane];
  const double W = L.ref.wsum;
  double r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
  if (W > 0.0 || W < 0.0) {
    const double inv_w = 1.0 / W;
    cx[0] = tot[0] * inv_w; cx[1] = tot[1] * inv_w; cx[2] = tot[2] * inv_w;
    cy[0] = L.ref.mean[0]; cy[1] = L.ref.mean[1]; cy[2] = L.ref.mean[2];
    if (!norotate) {
      double h[9];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) h[a * 3 + b] = tot[6 + a * 3 + b] - cx[a] * L.ref.sum_c[b];
      const double gx = tot[3] + tot[4] + tot[5] - (tot[0] * cx[0] + tot[1] * cx[1] + tot[2] * cx[2]);
      const QcpOut q = qcp_lambda(h, 0.5 * (gx + L.ref.gy));
      rotation_from_qcp(h, q.lambda, r);
    }
  }
  double* o = xf64 + f * kStatDoubles;
  for (int e = 0; e < 9; ++e) o[e] = r[e];
  for (int i = 0; i < 3; ++i) o[9 + i] = cy[i] - (r[i * 3 + 0] * cx[0] + r[i * 3 + 1] * cx[1] + r[i * 3 + 2] * cx[2]);
  if (xf32)
    for (int e = 0; e < 12; ++e) xf32[f * 12 + e] = (float)o[e];
}

// Every atom of every frame: out = R x + t.  Work items are (frame, 1024-atom
// chunk); each thread moves 4 atoms of a chunk, strided by the block size so
// that a warp's loads and stores cover contiguous 384-byte runs.
template <int STRIDE>
__global__ void __launch_bounds__(256) superpose_apply_kernel(const float* __restrict__ coords, int64_t n_frames,
                                                              int64_t n_atoms, const double* __restrict__ xf,
                                                              float* __restrict__ out) {
  constexpr int kChunk = 1024;
  const int64_t chunks = (n_atoms + kChunk - 1) / kChunk;
  const int64_t items = chunks * n_frames;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int64_t f = it / chunks;
    const int64_t a0 = (it - f * chunks) * kChunk;
    const double* x = xf + f * kStatDoubles;
    double R[9], t[3];
#pragma unroll
    for (int e = 0; e < 9; ++e) R[e] = __ldg(x + e);
    t[0] = __ldg(x + 9); t[1] = __ldg(x + 10); t[2] = __ldg(x + 11);
    const float* src = coords + (size_t)f * n_atoms * STRIDE;
    float* dst = out + (size_t)f * n_atoms * 3;
#pragma unroll
    for (int j = 0; j < kChunk / 256; ++j) {
      const int64_t a = a0 + threadIdx.x + j * 256;
      if (a < n_atoms) {
        const double p0 = __ldg(src + a * STRIDE + 0), p1 = __ldg(src + a * STRIDE + 1), p2 = __ldg(src + a * STRIDE + 2);
        dst[a * 3 + 0] = (float)(R[0] * p0 + R[1] * p1 + R[2] * p2 + t[0]);
        dst[a * 3 + 1] = (float)(R[3] * p0 + R[4] * p1 + R[5] * p2 + t[1]);
        dst[a * 3 + 2] = (float)(R[6] * p0 + R[7] * p1 + R[8] * p2 + t[2]);
      }
    }
  }
}

}  // namespace

cudaError_t launch_superpose_finalize(const FrameLaunch& L, int norotate, double* xf64, float* xf32, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((L.n_frames + 255) / 256);
  superpose_finalize_kernel<<<blocks, 256, 0, s>>>(L, frame_tiles(L), norotate, xf64, xf32);
  return cudaGetLastError();
}

cudaError_t launch_superpose_apply(const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                   const double* xf64, float* out, int sm_count, cudaStream_t s) {
  if (n_frames == 0 || n_atoms == 0) return cudaSuccess;
  const int64_t items = n_frames * ((n_atoms + 1023) / 1024);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * 8));
  if (stride == 4) superpose_apply_kernel<4><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, xf64, out);
  else superpose_apply_kernel<3><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, xf64, out);
  return cudaGetLastError();
}

}  // namespace wmd

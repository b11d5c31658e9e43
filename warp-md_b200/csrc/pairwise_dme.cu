// pairwise_dme.cu -- all-pairs distance-matrix error (PairwiseRmsdPlan metric
// "dme", crates/traj-engine/src/plans/rmsd/plan.rs:612-645).
//
// Per frame the reference lists the distances of every atom pair a < b of the
// selection (pair_distances_compact, plan.rs:1279-1302): the coordinate
// difference in f32, widened to f64, the minimum image per axis when a box is
// given (apply_pbc, crates/traj-core/src/pbc_math.rs:17-27), the distance in
// f64.  A frame pair (i, j) then gets sqrt(sum_k (d_i[k] - d_j[k])^2 / n_pairs),
// the sum in pair order, rounded to f32.
//
// Kernel.  A CTA per 32 x 32 tile of frame pairs (upper triangle only).  The
// K loop walks the atom pairs in the reference's order, 32 per step: the
// tile's 64 frames (32 row, 32 column) compute those 32 distances each into
// shared memory (FP64, in the reference's operation order, no contraction),
// then each thread adds (d_i - d_j)^2 for its 2 x 2 frame pairs.  Every thread
// walks k = 0, 1, 2, ... in order, so each sum is added in the reference's order
// and the results are bit-identical to it (the f32 frame coordinates are read
// as they are, without centring).  Distances are recomputed per tile rather
// than stored: an [n_frames][n_pairs] matrix is 8 * F * n(n-1)/2 bytes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_util.cuh"
#include "pairwise_dme.h"

namespace wmd {
namespace {

constexpr int kDmeTile = 32;     // frames per tile side
constexpr int kDmeK = 32;        // atom pairs per K step
constexpr int kDmeThreads = 256;  // 64 frames x 4 pair groups of 8 when filling; 2 x 2 frame pairs when adding

struct DmeArgs {
  const float* coords;
  int64_t F, n_atoms;
  int stride;
  const uint32_t* sel;
  int64_t n_sel, n_pairs;
  const float* box;
  float* out;
  int* status;
};

// pairs before row a: a (2n - a - 1) / 2
__device__ __forceinline__ int64_t row_start(int64_t a, int64_t n) { return a * (2 * n - a - 1) / 2; }

// atom pair k -> (a, b), a < b, lexicographic
__device__ __forceinline__ void pair_of(int64_t k, int64_t n, int64_t& a, int64_t& b) {
  const double m = (double)(2 * n - 1);
  int64_t r = (int64_t)((m - sqrt(m * m - 8.0 * (double)k)) * 0.5);
  r = max((int64_t)0, min(r, n - 2));
  while (r > 0 && row_start(r, n) > k) --r;
  while (r + 1 <= n - 2 && row_start(r + 1, n) <= k) ++r;
  a = r;
  b = k - row_start(r, n) + r + 1;
}

__device__ __forceinline__ double min_image(double d, double l) {
  // d -= round(d / l) * l, as two roundings (no fused multiply-add)
  return l > 0.0 ? __dsub_rn(d, __dmul_rn(round(__ddiv_rn(d, l)), l)) : d;
}

__global__ void __launch_bounds__(kDmeThreads) pair_dme_kernel(const DmeArgs A) {
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj < bi) return;  // lower triangle: mirrored from (bj, bi)
  __shared__ double dA[kDmeK][kDmeTile];
  __shared__ double dB[kDmeK][kDmeTile];
  const int tid = threadIdx.x;
  const int n_sel = (int)A.n_sel;
  // fill role: frame slot 0..63 (row frames, then column frames), 8 consecutive pairs
  const int fs = tid & 63;
  const int ps0 = (tid >> 6) * 8;
  const int64_t ff = fs < kDmeTile ? (int64_t)bi * kDmeTile + fs : (int64_t)bj * kDmeTile + (fs - kDmeTile);
  const bool fvalid = ff < A.F;
  const float* frame = A.coords + (size_t)(fvalid ? ff : 0) * A.n_atoms * A.stride;
  double lx = 0.0, ly = 0.0, lz = 0.0;
  if (A.box && fvalid) {
    lx = (double)A.box[ff * 3 + 0];
    ly = (double)A.box[ff * 3 + 1];
    lz = (double)A.box[ff * 3 + 2];
  }
  double(*dst)[kDmeTile] = fs < kDmeTile ? dA : dB;
  const int col = fs & (kDmeTile - 1);
  // add role: rows r0, r0 + 1 and columns c0, c0 + 1 of the tile
  const int r0 = 2 * (tid >> 4), c0 = 2 * (tid & 15);
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};

  for (int64_t k0 = 0; k0 < A.n_pairs; k0 += kDmeK) {
    {
      int64_t k = k0 + ps0;
      int64_t a = 0, b = 1;
      if (k < A.n_pairs) pair_of(k, n_sel, a, b);
#pragma unroll 1
      for (int u = 0; u < 8; ++u, ++k) {
        double dist = 0.0;
        if (k < A.n_pairs && fvalid) {
          int64_t ia = A.sel ? (int64_t)__ldg(A.sel + a) : a;
          int64_t ib = A.sel ? (int64_t)__ldg(A.sel + b) : b;
          if (ia >= A.n_atoms || ib >= A.n_atoms) {  // bad device-side selection: report, read atom 0
            atomicOr(A.status, kStatusBadIndex);
            ia = ia >= A.n_atoms ? 0 : ia;
            ib = ib >= A.n_atoms ? 0 : ib;
          }
          const float* pa = frame + ia * A.stride;
          const float* pb = frame + ib * A.stride;
          double dx = (double)__fsub_rn(__ldg(pb + 0), __ldg(pa + 0));
          double dy = (double)__fsub_rn(__ldg(pb + 1), __ldg(pa + 1));
          double dz = (double)__fsub_rn(__ldg(pb + 2), __ldg(pa + 2));
          if (A.box) {
            dx = min_image(dx, lx);
            dy = min_image(dy, ly);
            dz = min_image(dz, lz);
          }
          dist = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        }
        dst[ps0 + u][col] = dist;
        if (++b == n_sel) {
          ++a;
          b = a + 1;
        }
      }
    }
    __syncthreads();
    const int kn = (int)min((int64_t)kDmeK, A.n_pairs - k0);
#pragma unroll 4
    for (int kk = 0; kk < kn; ++kk) {
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y) {
          const double diff = __dsub_rn(dA[kk][r0 + x], dB[kk][c0 + y]);
          acc[x][y] = __dadd_rn(acc[x][y], __dmul_rn(diff, diff));
        }
    }
    __syncthreads();
  }

  const double np = (double)A.n_pairs;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) {
      const int64_t i = (int64_t)bi * kDmeTile + r0 + x, j = (int64_t)bj * kDmeTile + c0 + y;
      if (i >= A.F || j >= A.F) continue;
      if (i == j) {
        A.out[(size_t)i * A.F + i] = 0.f;
      } else if (i < j) {
        const float v = __double2float_rn(__dsqrt_rn(__ddiv_rn(acc[x][y], np)));
        A.out[(size_t)i * A.F + j] = v;
        A.out[(size_t)j * A.F + i] = v;
      }
    }
}

}  // namespace

cudaError_t launch_pair_dme(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                            int64_t n_sel, const float* box, float* out, int* status, cudaStream_t s) {
  if (n_frames == 0) return cudaSuccess;
  if (n_sel < 2) return cudaMemsetAsync(out, 0, (size_t)n_frames * n_frames * sizeof(float), s);
  DmeArgs a;
  a.coords = coords;
  a.F = n_frames;
  a.n_atoms = n_atoms;
  a.stride = stride;
  a.sel = sel;
  a.n_sel = n_sel;
  a.n_pairs = n_sel * (n_sel - 1) / 2;
  a.box = box;
  a.out = out;
  a.status = status;
  const int64_t nt = (n_frames + kDmeTile - 1) / kDmeTile;
  const dim3 grid((unsigned)nt, (unsigned)nt);
  pair_dme_kernel<<<grid, kDmeThreads, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace wmd

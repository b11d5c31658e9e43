// fluct.cu -- per-atom fluctuations over frames (RmsfPlan, AtomicFluctPlan,
// BfactorsPlan, AtomicAdpPlan) and per-group RMSD after superposition
// (RmsdPerResPlan).
//
// Fluctuations.  The reference keeps, per selected atom, a Welford running mean
// and M2 in FP64 on the host (crates/traj-engine/src/plans/geometry/rms.rs:
// 96-218), or sums x, y, z and |x|^2 (rms.rs:397-429 for the 6 ADP moments).
// Here every atom's coordinates are shifted by their value in the first frame
// (differences of two floats are exact in FP64, and so are their squares), and
// the nine moments sum d, sum d_c^2, sum d_x d_y / d_x d_z / d_y d_z run in FP64:
//   * fluct_partial_kernel: a thread per selected atom and frame group -- a
//     CTA covers 256 consecutive selected atoms over one contiguous run of
//     frames, so a warp's three loads per frame cover 384 contiguous bytes of
//     a dense selection; partial moments go to [group][atom][9];
//   * fluct_reduce_kernel adds the groups in order into a running FP64
//     accumulator (host-resident trajectories arrive chunk by chunk);
//   * fluct_finalize_kernel turns the moments into RMSF and the ADP tensor.
//
// Per-group RMSD.  Per frame, the selection's transform (R, t) comes from the
// superposition path; |R x + t - y|^2 against the all-atom reference is summed
// per group in FP64 (rms.rs:633-671), see group_rmsd_kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_util.cuh"
#include "fluct.h"
#include "wmd_internal.h"

namespace wmd {
namespace {

constexpr int kFluctThreads = 256;

template <int STRIDE>
__global__ void __launch_bounds__(kFluctThreads) fluct_shift_kernel(const float* __restrict__ coords,
                                                                    int64_t n_atoms, const uint32_t* __restrict__ sel,
                                                                    int64_t n_sel, float* __restrict__ shift,
                                                                    int* status) {
  const int64_t i = (int64_t)blockIdx.x * kFluctThreads + threadIdx.x;
  if (i >= n_sel) return;
  int64_t a = sel ? (int64_t)sel[i] : i;
  if (a >= n_atoms) {  // bad device-side selection: report, read atom 0
    atomicOr(status, kStatusBadIndex);
    a = 0;
  }
  for (int c = 0; c < 3; ++c) shift[i * 3 + c] = coords[a * STRIDE + c];
}

template <int STRIDE>
__global__ void __launch_bounds__(kFluctThreads) fluct_partial_kernel(const float* __restrict__ coords,
                                                                      int64_t n_frames, int64_t n_atoms,
                                                                      const uint32_t* __restrict__ sel, int64_t n_sel,
                                                                      const float* __restrict__ shift,
                                                                      double* __restrict__ part) {
  const int64_t i = (int64_t)blockIdx.x * kFluctThreads + threadIdx.x;
  const int g = blockIdx.y, G = gridDim.y;
  if (i >= n_sel) return;
  const int64_t f0 = n_frames * g / G, f1 = n_frames * (g + 1) / G;
  int64_t a = sel ? (int64_t)sel[i] : i;
  if (a >= n_atoms) a = 0;  // reported by fluct_shift_kernel
  const float s0 = shift[i * 3 + 0], s1 = shift[i * 3 + 1], s2 = shift[i * 3 + 2];
  double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const float* p = coords + (size_t)f0 * n_atoms * STRIDE + a * STRIDE;
  const size_t step = (size_t)n_atoms * STRIDE;
  int64_t f = f0;
  for (; f + 4 <= f1; f += 4) {
    float x[4][3];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x[u][0] = __ldg(p + u * step + 0); x[u][1] = __ldg(p + u * step + 1); x[u][2] = __ldg(p + u * step + 2);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double d0 = (double)x[u][0] - s0, d1 = (double)x[u][1] - s1, d2 = (double)x[u][2] - s2;
      m[0] += d0; m[1] += d1; m[2] += d2;
      m[3] = fma(d0, d0, m[3]); m[4] = fma(d1, d1, m[4]); m[5] = fma(d2, d2, m[5]);
      m[6] = fma(d0, d1, m[6]); m[7] = fma(d0, d2, m[7]); m[8] = fma(d1, d2, m[8]);
    }
    p += 4 * step;
  }
  for (; f < f1; ++f) {
    const double d0 = (double)__ldg(p) - s0, d1 = (double)__ldg(p + 1) - s1, d2 = (double)__ldg(p + 2) - s2;
    m[0] += d0; m[1] += d1; m[2] += d2;
    m[3] = fma(d0, d0, m[3]); m[4] = fma(d1, d1, m[4]); m[5] = fma(d2, d2, m[5]);
    m[6] = fma(d0, d1, m[6]); m[7] = fma(d0, d2, m[7]); m[8] = fma(d1, d2, m[8]);
    p += step;
  }
  double* o = part + ((size_t)g * n_sel + i) * kFluctMoments;
#pragma unroll
  for (int e = 0; e < 9; ++e) o[e] = m[e];
}

__global__ void __launch_bounds__(kFluctThreads) fluct_reduce_kernel(const double* __restrict__ part, int G,
                                                                     int64_t n_sel, double* __restrict__ acc) {
  const int64_t i = (int64_t)blockIdx.x * kFluctThreads + threadIdx.x;
  if (i >= n_sel) return;
  double m[9];
  for (int e = 0; e < 9; ++e) m[e] = acc[i * kFluctMoments + e];
  for (int g = 0; g < G; ++g)
    for (int e = 0; e < 9; ++e) m[e] += part[((size_t)g * n_sel + i) * kFluctMoments + e];
  for (int e = 0; e < 9; ++e) acc[i * kFluctMoments + e] = m[e];
}

// RMSF = sqrt(max(sum_c var_c, 0)) (rms.rs:199-212); ADP = (uxx, uyy, uzz, uxy,
// uxz, uyz) with the diagonal clamped at 0 (rms.rs:384-406).  Both are
// invariant under the per-atom shift.
__global__ void __launch_bounds__(kFluctThreads) fluct_finalize_kernel(const double* __restrict__ acc, int64_t n_sel,
                                                                       int64_t n_frames, float* __restrict__ rmsf,
                                                                       float* __restrict__ adp) {
  const int64_t i = (int64_t)blockIdx.x * kFluctThreads + threadIdx.x;
  if (i >= n_sel) return;
  const double* m = acc + i * kFluctMoments;
  const double inv = 1.0 / (double)n_frames;
  const double mx = m[0] * inv, my = m[1] * inv, mz = m[2] * inv;
  const double vx = m[3] * inv - mx * mx, vy = m[4] * inv - my * my, vz = m[5] * inv - mz * mz;
  if (rmsf) {
    const double var = vx + vy + vz;
    rmsf[i] = (float)sqrt(var > 0.0 ? var : 0.0);
  }
  if (adp) {
    float* o = adp + i * 6;
    o[0] = (float)(vx > 0.0 ? vx : 0.0);
    o[1] = (float)(vy > 0.0 ? vy : 0.0);
    o[2] = (float)(vz > 0.0 ? vz : 0.0);
    o[3] = (float)(m[6] * inv - mx * my);
    o[4] = (float)(m[7] * inv - mx * mz);
    o[5] = (float)(m[8] * inv - my * mz);
  }
}

// Per-group RMSD.  Groups are contiguous ranges of the concatenated atom list
// and are packed, in order, into blocks of at most kGroupTile list positions
// (a larger group gets a block of its own, walked in tiles).  A CTA takes a
// (frame, block) item: its threads compute |R x + t - y|^2 for consecutive list
// positions -- coalesced loads when a residue's atoms are consecutive -- into
// shared memory, then one thread per group adds its range in list order (the
// order of the reference's loop), so results are deterministic.
constexpr int kGroupTile = 2048;

// CONTIG: the concatenated atom list is a run of consecutive atoms (list
// position q is atom contig_base + q), so no index load precedes the
// coordinate loads.
template <int STRIDE, bool CONTIG>
__global__ void __launch_bounds__(256, 4) group_rmsd_kernel(const float* __restrict__ coords, int64_t n_frames,
                                                         int64_t n_atoms, const double* __restrict__ xf,
                                                         const uint32_t* __restrict__ goff,
                                                         const uint32_t* __restrict__ gatoms, int64_t contig_base,
                                                         const uint32_t* __restrict__ blocks, int64_t n_blocks,
                                                         int64_t n_groups, const float* __restrict__ ref_all,
                                                         float* __restrict__ out) {
  __shared__ double sq[kGroupTile];
  __shared__ double rt[12];
  const int tid = threadIdx.x;
  const int64_t items = n_frames * n_blocks;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int64_t f = it / n_blocks, b = it - f * n_blocks;
    const uint32_t g0 = blocks[b], g1 = blocks[b + 1];
    const uint32_t p0 = goff[g0], p1 = goff[g1];
    if (tid < 12) rt[tid] = xf ? __ldg(xf + f * kStatDoubles + tid) : ((tid == 0 || tid == 4 || tid == 8) ? 1.0 : 0.0);
    __syncthreads();
    const float* frame = coords + (size_t)f * n_atoms * STRIDE;
    // a block spans several tiles only when it is one group larger than a tile
    double big = 0.0;
    for (uint32_t q0 = p0; q0 < p1; q0 += kGroupTile) {
      const uint32_t q1 = min(p1, q0 + (uint32_t)kGroupTile);
      {
        double R[9], t[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) R[e] = rt[e];
        t[0] = rt[9]; t[1] = rt[10]; t[2] = rt[11];
        // 4 positions per thread per pass: all loads issued before any use
        for (uint32_t qb = q0; qb < q1; qb += 4 * 256) {
          float xv[4][3], yv[4][3];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint32_t q = qb + tid + u * 256;
            if (q < q1) {
              const int64_t a = CONTIG ? contig_base + q : (int64_t)__ldg(gatoms + q);
              xv[u][0] = __ldg(frame + a * STRIDE); xv[u][1] = __ldg(frame + a * STRIDE + 1);
              xv[u][2] = __ldg(frame + a * STRIDE + 2);
              yv[u][0] = __ldg(ref_all + a * 3); yv[u][1] = __ldg(ref_all + a * 3 + 1);
              yv[u][2] = __ldg(ref_all + a * 3 + 2);
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint32_t q = qb + tid + u * 256;
            if (q < q1) {
              const double x0 = xv[u][0], x1 = xv[u][1], x2 = xv[u][2];
              const double d0 = R[0] * x0 + R[1] * x1 + R[2] * x2 + t[0] - (double)yv[u][0];
              const double d1 = R[3] * x0 + R[4] * x1 + R[5] * x2 + t[1] - (double)yv[u][1];
              const double d2 = R[6] * x0 + R[7] * x1 + R[8] * x2 + t[2] - (double)yv[u][2];
              sq[q - q0] = d0 * d0 + d1 * d1 + d2 * d2;
            }
          }
        }
      }
      __syncthreads();
      if (g1 - g0 == 1 && p1 - p0 > (uint32_t)kGroupTile) {
        // one large group: thread 0 adds the tile in list order
        if (tid == 0)
          for (uint32_t q = q0; q < q1; ++q) big += sq[q - q0];
      } else {
        for (uint32_t g = g0 + tid; g < g1; g += 256) {
          const uint32_t a0 = goff[g], a1 = goff[g + 1];
          double acc = 0.0;
          for (uint32_t q = a0; q < a1; ++q) acc += sq[q - q0];
          out[f * n_groups + g] = (float)sqrt(acc / (a1 > a0 ? (double)(a1 - a0) : 1.0));
        }
      }
      __syncthreads();
    }
    if (g1 - g0 == 1 && p1 - p0 > (uint32_t)kGroupTile && tid == 0)
      out[f * n_groups + g0] = (float)sqrt(big / (double)(p1 - p0));
    if (p1 == p0)  // blocks of empty groups only
      for (uint32_t g = g0 + tid; g < g1; g += 256) out[f * n_groups + g] = 0.f;
    __syncthreads();  // rt is rewritten by the next item
  }
}

}  // namespace

// Frame groups: the count whose blocks fill whole waves of resident CTAs best
// (a partial last wave leaves SMs idle while the HBM stream is the bound),
// at least 16 frames per group.
int fluct_groups(int64_t n_sel, int64_t n_frames, int sm_count) {
  static int occ = 0;
  if (occ == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fluct_partial_kernel<3>, kFluctThreads, 0) != cudaSuccess)
      b = 8;
    occ = std::max(b, 1);
  }
  const int64_t blocks = std::max<int64_t>(1, (n_sel + kFluctThreads - 1) / kFluctThreads);
  const int64_t cap = (int64_t)sm_count * occ;
  const int64_t g_max = std::max<int64_t>(1, std::min<int64_t>(1024, n_frames / 16));
  int64_t best = 1;
  double best_eff = -1.0;
  for (int64_t G = 1; G <= g_max && G <= 64; ++G) {
    const int64_t total = blocks * G;
    const int64_t waves = (total + cap - 1) / cap;
    const double eff = (double)total / (double)(waves * cap);
    if (eff > best_eff + 1e-9) {
      best = G;
      best_eff = eff;
    }
    if (eff > 0.95 && total >= cap) break;  // first full wave at 95 %
  }
  return (int)best;
}

cudaError_t launch_fluct_shift(const float* coords, int64_t n_atoms, int stride, const uint32_t* sel, int64_t n_sel,
                               float* shift, int* status, cudaStream_t s) {
  if (n_sel == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n_sel + kFluctThreads - 1) / kFluctThreads);
  if (stride == 4) fluct_shift_kernel<4><<<blocks, kFluctThreads, 0, s>>>(coords, n_atoms, sel, n_sel, shift, status);
  else fluct_shift_kernel<3><<<blocks, kFluctThreads, 0, s>>>(coords, n_atoms, sel, n_sel, shift, status);
  return cudaGetLastError();
}

cudaError_t launch_fluct_chunk(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                               int64_t n_sel, const float* shift, int groups, double* part, double* acc,
                               cudaStream_t s) {
  if (n_sel == 0 || n_frames == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n_sel + kFluctThreads - 1) / kFluctThreads);
  const dim3 grid(blocks, (unsigned)groups);
  if (stride == 4)
    fluct_partial_kernel<4><<<grid, kFluctThreads, 0, s>>>(coords, n_frames, n_atoms, sel, n_sel, shift, part);
  else
    fluct_partial_kernel<3><<<grid, kFluctThreads, 0, s>>>(coords, n_frames, n_atoms, sel, n_sel, shift, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  fluct_reduce_kernel<<<blocks, kFluctThreads, 0, s>>>(part, groups, n_sel, acc);
  return cudaGetLastError();
}

cudaError_t launch_fluct_finalize(const double* acc, int64_t n_sel, int64_t n_frames, float* rmsf, float* adp,
                                  cudaStream_t s) {
  if (n_sel == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n_sel + kFluctThreads - 1) / kFluctThreads);
  fluct_finalize_kernel<<<blocks, kFluctThreads, 0, s>>>(acc, n_sel, n_frames, rmsf, adp);
  return cudaGetLastError();
}

int group_blocks(const uint32_t* goff, int64_t n_groups, uint32_t* blocks) {
  // greedy, in order: a block ends before the group that would take it past
  // kGroupTile positions or kGroupTile groups
  int64_t nb = 0;
  blocks[0] = 0;
  int64_t g = 0;
  while (g < n_groups) {
    const uint32_t start = goff[g];
    int64_t h = g + 1;
    while (h < n_groups && goff[h + 1] - start <= (uint32_t)kGroupTile && h - g < kGroupTile) ++h;
    blocks[++nb] = (uint32_t)h;
    g = h;
  }
  return (int)nb;
}

cudaError_t launch_group_rmsd(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const double* xf,
                              const uint32_t* goff, const uint32_t* gatoms, int64_t contig_base,
                              const uint32_t* blocks, int64_t n_blocks, int64_t n_groups, const float* ref_all,
                              float* out, int sm_count, cudaStream_t s) {
  if (n_frames == 0 || n_groups == 0) return cudaSuccess;
  const int64_t items = n_frames * n_blocks;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * 8));
#define WMD_GROUP_LAUNCH(ST, CG)                                                                                 \
  group_rmsd_kernel<ST, CG><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, xf, goff, gatoms, contig_base, blocks, \
                                                 n_blocks, n_groups, ref_all, out)
  const bool contig = contig_base >= 0;
  if (stride == 4) {
    if (contig) WMD_GROUP_LAUNCH(4, true);
    else WMD_GROUP_LAUNCH(4, false);
  } else {
    if (contig) WMD_GROUP_LAUNCH(3, true);
    else WMD_GROUP_LAUNCH(3, false);
  }
#undef WMD_GROUP_LAUNCH
  return cudaGetLastError();
}

}  // namespace wmd

// batched.cu -- per-frame RMSD (+ dRMSD/dx) of many trajectories of uneven
// size in one launch sequence.
//
// The reference runs one plan per trajectory, serially (no batched form).
// Here all trajectories' (atom tile, frame) work items form one global list,
// trajectory-major and tile-major inside a trajectory; persistent CTAs each
// take a contiguous, balanced run of items and walk it with incremental
// (trajectory, tile, frame) cursors, so a 50-atom trajectory and a 20,000-atom
// one share the same launch without padding.  The per-item streaming and the
// FP64 statistics are those of the single-trajectory kernel (rmsd_frames.cu):
// 1-D bulk copies into a shared-memory ring, reference tile in registers,
// butterfly reduce-scatter, one 16-double partial per item.  Frames are then
// finished (QCP) by a warp each, near-zero RMSDs get the explicit residual
// pass, and with gradients a prologue derives R from the QCP eigenvector and
// a second streaming pass writes dRMSD/dx.
//
// wmd_batched_prepare sizes every buffer, uploads the trajectory table and
// picks the tile shape (512- or 1024-atom tiles) by timing both on the batch;
// wmd_batched_rmsd then only enqueues kernels on the stream (no allocation, no
// host synchronisation), so it can be captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/warpmd_rmsd.h"
#include "batched.h"
#include "device_util.cuh"
#include "qcp.cuh"
#include "wmd_internal.h"

namespace wmd {
namespace {

enum BMode : int { kBFwd = 0, kBBwd = 1 };

template <int APT>
struct BGeo {
  static constexpr int kTile = kConsumerThreads * APT;
  static constexpr int kStageBytes = ((kTile * 3 * 4 + 32) + 127) / 128 * 128;
  static constexpr int kStagesRaw = 51200 / kStageBytes;
  static constexpr int kStages = kStagesRaw < 3 ? 3 : (kStagesRaw > 8 ? 8 : kStagesRaw);
  static constexpr int kBarOffset = kStages * kStageBytes;
  static constexpr int kRedOffset = kBarOffset + kStages * 8;
  static constexpr int kAbortOffset = kRedOffset + 2 * kConsumerWarps * 16 * 8;
  static constexpr int kSmemBytes = kAbortOffset + 16;
};

// index of the segment containing global position `x` of a prefix array
__device__ __forceinline__ int seg_of(const BatchSeg* segs, int n, int64_t x, bool by_frame) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int64_t v = by_frame ? segs[mid].frame0 : segs[mid].item0;
    if (v <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct Cursor {
  int seg;
  int t;
  int64_t f;
};

__device__ __forceinline__ void cursor_init(const BatchLaunch& B, int64_t w, Cursor& c) {
  c.seg = seg_of(B.segs, B.n_segs, w, false);
  // skip empty segments sharing the same item0
  while (c.seg + 1 < B.n_segs && B.segs[c.seg + 1].item0 <= w) ++c.seg;
  const BatchSeg& s = B.segs[c.seg];
  const int64_t l = w - s.item0;
  c.t = s.n_frames > 0 ? (int)(l / s.n_frames) : 0;
  c.f = l - (int64_t)c.t * s.n_frames;
}

__device__ __forceinline__ void cursor_next(const BatchLaunch& B, Cursor& c) {
  const BatchSeg& s = B.segs[c.seg];
  if (++c.f == s.n_frames) {
    c.f = 0;
    if (++c.t == s.n_tiles) {
      c.t = 0;
      do {
        ++c.seg;
      } while (c.seg < B.n_segs && (B.segs[c.seg].n_frames == 0 || B.segs[c.seg].n_tiles == 0));
    }
  }
}

template <int APT>
__device__ __forceinline__ void batched_issue(const BatchSeg& s, int t, int64_t f, unsigned char* dst, uint64_t* bar) {
  constexpr int T = BGeo<APT>::kTile;
  const int64_t a0 = (int64_t)t * T;
  const int64_t a1 = min(s.n_atoms, a0 + T);
  const unsigned char* base = reinterpret_cast<const unsigned char*>(s.coords);
  const uint64_t total_al = ((uint64_t)s.n_frames * (uint64_t)s.n_atoms * 12ull) & ~15ull;
  const uint64_t b0 = (uint64_t)(f * s.n_atoms + a0) * 12ull;
  const uint64_t b1 = (uint64_t)(f * s.n_atoms + a1) * 12ull;
  const uint64_t c0 = b0 & ~15ull;
  uint64_t c1 = (b1 + 15ull) & ~15ull;
  if (c1 > total_al) {
    const uint64_t tail0 = total_al > c0 ? total_al : c0;
    for (uint64_t bb = tail0; bb < b1; bb += 4)
      *reinterpret_cast<float*>(dst + (bb - c0)) = __ldg(reinterpret_cast<const float*>(base + bb));
    c1 = tail0;
  }
  const uint32_t core = (uint32_t)(c1 - c0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_arrive_expect_tx(bar, core);
  if (core) bulk_copy_g2s(dst, base + c0, core, bar);
}

template <int APT, int MODE>
__global__ void __launch_bounds__(kThreads, 3) batched_stream_kernel(const BatchLaunch B) {
  using G = BGeo<APT>;
  constexpr int T = G::kTile;
  constexpr int S = G::kStages;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::kBarOffset);
  double* red = reinterpret_cast<double*>(smem + G::kRedOffset);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::kAbortOffset);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t W = B.total_items;
  const int64_t w0 = W * blockIdx.x / gridDim.x, w1 = W * (blockIdx.x + 1) / gridDim.x;
  const int64_t n_items = w1 - w0;
  if (tid == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&full[st], 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (n_items <= 0) return;

  Cursor pc;  // producer cursor (thread 0)
  int64_t issued = 0;
  if (tid == 0) {
    cursor_init(B, w0, pc);
    for (; issued < S - 1 && issued < n_items; ++issued) {
      batched_issue<APT>(B.segs[pc.seg], pc.t, pc.f, smem + (issued % S) * G::kStageBytes, &full[issued % S]);
      cursor_next(B, pc);
    }
  }
  Cursor c;
  cursor_init(B, w0, c);
  int cur_seg = -1, cur_tile = -1;
  double yr[APT][3];
  int s = 0;
  uint32_t phase = 0;
  for (int64_t i = 0; i < n_items; ++i) {
    if (tid == 0 && issued < n_items) {
      const int sp = (int)(issued % S);
      batched_issue<APT>(B.segs[pc.seg], pc.t, pc.f, smem + sp * G::kStageBytes, &full[sp]);
      ++issued;
      cursor_next(B, pc);
    }
    const BatchSeg& sg = B.segs[c.seg];
    const int64_t a0 = (int64_t)c.t * T;
    const int len = (int)(min(sg.n_atoms, a0 + T) - a0);
    if (c.seg != cur_seg || c.t != cur_tile) {
      cur_seg = c.seg;
      cur_tile = c.t;
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        const int k = tid + j * kConsumerThreads;
        if (k < len) {
          const double* y = sg.yc + (a0 + k) * 3;
          yr[j][0] = y[0]; yr[j][1] = y[1]; yr[j][2] = y[2];
        } else {
          yr[j][0] = yr[j][1] = yr[j][2] = 0.0;
        }
      }
    }
    const bool ok = mbar_wait(&full[s], phase, B.status, kStatusTimeoutFull, abort_flag);
    const float* xs = reinterpret_cast<const float*>(smem + s * G::kStageBytes) +
                      (int)(((uint64_t)(c.f * sg.n_atoms + a0) * 3) & 3ull);
    const int64_t gitem = w0 + i;
    if (MODE == kBBwd) {
      if (ok) {
        const double* rt = B.rot + (sg.frame0 + c.f) * kStatDoubles;
        double R[9], cc[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) R[e] = rt[e];
        cc[0] = rt[9]; cc[1] = rt[10]; cc[2] = rt[11];
        const double scale = sg.grad ? rt[12] : 0.0;
        float* gframe = sg.grad ? sg.grad + (size_t)c.f * sg.n_atoms * 3 : nullptr;
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          const int k = tid + j * kConsumerThreads;
          if (gframe && k < len) {
            const float x0 = xs[k * 3 + 0], x1 = xs[k * 3 + 1], x2 = xs[k * 3 + 2];
            const double ty0 = R[0] * yr[j][0] + R[3] * yr[j][1] + R[6] * yr[j][2];
            const double ty1 = R[1] * yr[j][0] + R[4] * yr[j][1] + R[7] * yr[j][2];
            const double ty2 = R[2] * yr[j][0] + R[5] * yr[j][1] + R[8] * yr[j][2];
            float* g = gframe + (size_t)(a0 + k) * 3;
            g[0] = (float)(scale * (((double)x0 - cc[0]) - ty0));
            g[1] = (float)(scale * (((double)x1 - cc[1]) - ty1));
            g[2] = (float)(scale * (((double)x2 - cc[2]) - ty2));
          }
        }
      }
      named_barrier_sync(1, kConsumerThreads);
    } else {
      double acc[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[e] = 0.0;
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        const int k = tid + j * kConsumerThreads;
        const bool in = ok && k < len;
        const double x0 = in ? (double)xs[k * 3 + 0] : 0.0;
        const double x1 = in ? (double)xs[k * 3 + 1] : 0.0;
        const double x2 = in ? (double)xs[k * 3 + 2] : 0.0;
        acc[0] += x0; acc[1] += x1; acc[2] += x2;
        acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
        acc[6] = fma(x0, yr[j][0], acc[6]);  acc[7] = fma(x0, yr[j][1], acc[7]);  acc[8] = fma(x0, yr[j][2], acc[8]);
        acc[9] = fma(x1, yr[j][0], acc[9]);  acc[10] = fma(x1, yr[j][1], acc[10]); acc[11] = fma(x1, yr[j][2], acc[11]);
        acc[12] = fma(x2, yr[j][0], acc[12]); acc[13] = fma(x2, yr[j][1], acc[13]); acc[14] = fma(x2, yr[j][2], acc[14]);
      }
      const double v = warp_reduce_scatter16(acc);
      double* rb = red + (i & 1) * (kConsumerWarps * 16);
      if ((lane & 1) == 0) rb[warp * 16 + (lane >> 1)] = v;
      named_barrier_sync(1, kConsumerThreads);
      if (warp == (int)(i & (kConsumerWarps - 1)) && lane < 16) {
        double tot = 0.0;
#pragma unroll
        for (int wv = 0; wv < kConsumerWarps; ++wv) tot += rb[wv * 16 + lane];
        B.partial[(size_t)gitem * kStatDoubles + lane] = tot;
      }
    }
    if (*abort_flag) break;
    if (++s == S) { s = 0; phase ^= 1u; }
    cursor_next(B, c);
  }
  if (tid == 0) {
    const int64_t first = issued > S ? issued - S : 0;
    for (int64_t j = first; j < issued; ++j) {
      const int st = (int)(j % S);
      const uint32_t ph = (uint32_t)((j / S) & 1);
      const uint64_t t0 = global_timer_ns();
      while (!mbar_try_wait(&full[st], ph)) {
        if (global_timer_ns() - t0 > kWaitLimitNs) {
          atomicOr(B.status, kStatusTimeoutDrain);
          break;
        }
      }
    }
  }
}

// One CTA per trajectory: y_c = y - mean(y) into the workspace, and the
// statistics the finisher needs (sum of y_c, G_y), in fixed-order trees.
__global__ void __launch_bounds__(256) batched_ref_prep(BatchSeg* segs) {
  __shared__ double red[8][3];
  __shared__ double bc[3];
  BatchSeg& s = segs[blockIdx.x];
  const float* ref = s.ref;
  double* yc = s.yc;
  const int64_t n = s.n_atoms;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto sum3 = [&](double& a, double& b, double& c) {
    for (int o = 16; o; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) { red[warp][0] = a; red[warp][1] = b; red[warp][2] = c; }
    __syncthreads();
    if (tid == 0) {
      double s0 = 0, s1 = 0, s2 = 0;
      for (int w = 0; w < 8; ++w) { s0 += red[w][0]; s1 += red[w][1]; s2 += red[w][2]; }
      bc[0] = s0; bc[1] = s1; bc[2] = s2;
    }
    __syncthreads();
    a = bc[0]; b = bc[1]; c = bc[2];
    __syncthreads();
  };
  if (n == 0 || s.n_frames == 0) return;
  double m0 = 0, m1 = 0, m2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) { m0 += ref[k * 3]; m1 += ref[k * 3 + 1]; m2 += ref[k * 3 + 2]; }
  sum3(m0, m1, m2);
  const double inv = 1.0 / (double)n;
  m0 *= inv; m1 *= inv; m2 *= inv;
  double c0 = 0, c1 = 0, c2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) {
    const double a = (double)ref[k * 3] - m0, b = (double)ref[k * 3 + 1] - m1, c = (double)ref[k * 3 + 2] - m2;
    yc[k * 3] = a; yc[k * 3 + 1] = b; yc[k * 3 + 2] = c;
    c0 += a; c1 += b; c2 += c;
  }
  sum3(c0, c1, c2);
  double g0 = 0, g1 = 0, g2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) {
    const double a = yc[k * 3] - c0 * inv, b = yc[k * 3 + 1] - c1 * inv, c = yc[k * 3 + 2] - c2 * inv;
    g0 += a * a; g1 += b * b; g2 += c * c;
  }
  sum3(g0, g1, g2);
  if (tid == 0) {
    s.sum_c[0] = c0; s.sum_c[1] = c1; s.sum_c[2] = c2;
    s.gy = g0 + g1 + g2;
  }
}

// One warp per frame of the batch: partials in tile order, QCP, outputs.
__global__ void __launch_bounds__(256) batched_finalize(const BatchLaunch B) {
  const int64_t g = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (g >= B.total_frames) return;
  const int lane = threadIdx.x & 31;
  const BatchSeg& sg = B.segs[seg_of(B.segs, B.n_segs, g, true)];
  const int64_t f = g - sg.frame0;
  double s = 0.0;
  if (lane < 16)
    for (int t = 0; t < sg.n_tiles; ++t) s += B.partial[(size_t)(sg.item0 + (int64_t)t * sg.n_frames + f) * kStatDoubles + lane];
  double tot[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) tot[e] = __shfl_sync(0xffffffffu, s, e);
  if (lane != 0) return;
  if (sg.n_atoms == 0) {
    // empty selection: RMSD 0, no rotation (the single-trajectory path writes the same)
    sg.rmsd[f] = 0.0;
    if (B.stats)
      for (int e = 0; e < 16; ++e) B.stats[g * kStatDoubles + e] = 0.0;
    return;
  }
  const double n = (double)sg.n_atoms, inv_n = 1.0 / n;
  const double sx[3] = {tot[0], tot[1], tot[2]};
  double h[9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) h[a * 3 + b] = tot[6 + a * 3 + b] - sx[a] * sg.sum_c[b] * inv_n;
  const double gx = tot[3] + tot[4] + tot[5] - (sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]) * inv_n;
  const QcpOut q = qcp_lambda(h, 0.5 * (gx + sg.gy));
  const double rmsd = sqrt(msd_from(gx, sg.gy, q.lambda, n));
  sg.rmsd[f] = rmsd;
  if (B.stats) {
    double* st = B.stats + g * kStatDoubles;
    st[0] = sx[0] * inv_n; st[1] = sx[1] * inv_n; st[2] = sx[2] * inv_n;
    for (int e = 0; e < 9; ++e) st[3 + e] = h[e];
    st[12] = q.lambda; st[13] = rmsd; st[14] = n; st[15] = gx + sg.gy;
  }
  if (rmsd < kRefineScale * (gx + sg.gy) * inv_n) {
    const unsigned slot = atomicAdd(B.refine_count, 1u);
    double* rec = B.refine + (size_t)slot * kStatDoubles;
    rec[0] = (double)g;
    rec[1] = sx[0] * inv_n; rec[2] = sx[1] * inv_n; rec[3] = sx[2] * inv_n;
    for (int e = 0; e < 9; ++e) rec[4 + e] = h[e];
    rec[13] = q.lambda;
  }
}

// Explicit residual pass for the batch's near-zero RMSD frames.
__global__ void __launch_bounds__(256) batched_refine(const BatchLaunch B) {
  __shared__ double sh[12];
  __shared__ double red[8];
  const unsigned count = *B.refine_count;
  for (unsigned r = blockIdx.x; r < count; r += gridDim.x) {
    const double* rec = B.refine + (size_t)r * kStatDoubles;
    const int64_t g = (int64_t)rec[0];
    const BatchSeg& sg = B.segs[seg_of(B.segs, B.n_segs, g, true)];
    const int64_t f = g - sg.frame0;
    if (threadIdx.x == 0) {
      double h[9], R[9];
      for (int e = 0; e < 9; ++e) h[e] = rec[4 + e];
      rotation_from_qcp(h, rec[13], R);
      for (int e = 0; e < 9; ++e) sh[e] = R[e];
      sh[9] = rec[1]; sh[10] = rec[2]; sh[11] = rec[3];
    }
    __syncthreads();
    const double inv_n = 1.0 / (double)sg.n_atoms;
    const double my0 = sg.sum_c[0] * inv_n, my1 = sg.sum_c[1] * inv_n, my2 = sg.sum_c[2] * inv_n;
    const float* frame = sg.coords + (size_t)f * sg.n_atoms * 3;
    double acc = 0.0;
    for (int64_t k = threadIdx.x; k < sg.n_atoms; k += blockDim.x) {
      const double d0 = (double)frame[k * 3] - sh[9], d1 = (double)frame[k * 3 + 1] - sh[10],
                   d2 = (double)frame[k * 3 + 2] - sh[11];
      const double r0 = sh[0] * d0 + sh[1] * d1 + sh[2] * d2 - (sg.yc[k * 3] - my0);
      const double r1 = sh[3] * d0 + sh[4] * d1 + sh[5] * d2 - (sg.yc[k * 3 + 1] - my1);
      const double r2 = sh[6] * d0 + sh[7] * d1 + sh[8] * d2 - (sg.yc[k * 3 + 2] - my2);
      acc += r0 * r0 + r1 * r1 + r2 * r2;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += red[w];
      const double rmsd = sqrt(t * inv_n);
      sg.rmsd[f] = rmsd;
      if (B.stats) B.stats[g * kStatDoubles + 13] = rmsd;
    }
    __syncthreads();
  }
}

// Per frame: R from the QCP eigenvector, centroid, 1 / (n rmsd).
__global__ void batched_bwd_prologue(const BatchLaunch B) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= B.total_frames) return;
  const double* st = B.stats + g * kStatDoubles;
  double h[9], r[9];
  for (int e = 0; e < 9; ++e) h[e] = st[3 + e];
  rotation_from_qcp(h, st[12], r);
  const double rmsd = st[13], n = st[14];
  double* o = B.rot + g * kStatDoubles;
  for (int e = 0; e < 9; ++e) o[e] = r[e];
  o[9] = st[0]; o[10] = st[1]; o[11] = st[2];
  o[12] = (rmsd > 0.0 && n > 0.0) ? 1.0 / (n * rmsd) : 0.0;
}

template <int APT, int MODE>
cudaError_t launch_stream(const BatchLaunch& B, int grid, cudaStream_t s) {
  auto kern = batched_stream_kernel<APT, MODE>;
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, BGeo<APT>::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  kern<<<grid, kThreads, BGeo<APT>::kSmemBytes, s>>>(B);
  return cudaGetLastError();
}

template <int APT, int MODE>
int occupancy_of() {
  auto kern = batched_stream_kernel<APT, MODE>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, BGeo<APT>::kSmemBytes);
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kThreads, BGeo<APT>::kSmemBytes) != cudaSuccess)
    blocks = 1;
  return blocks < 1 ? 1 : blocks;
}

}  // namespace

int batched_tile_atoms(int apt) { return kConsumerThreads * apt; }

cudaError_t batched_enqueue(const BatchPlan& P, bool with_grad, cudaStream_t s) {
  BatchLaunch B = P.launch;
  cudaError_t e;
  batched_ref_prep<<<P.n_segs, 256, 0, s>>>(P.segs_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(B.refine_count, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
  if (B.total_items > 0) {
    e = P.apt == 4 ? launch_stream<4, kBFwd>(B, P.grid_fwd, s) : launch_stream<8, kBFwd>(B, P.grid_fwd, s);
    if (e != cudaSuccess) return e;
  }
  if (B.total_frames > 0) {
    batched_finalize<<<(unsigned)((B.total_frames + 7) / 8), 256, 0, s>>>(B);
    batched_refine<<<(unsigned)std::min<int64_t>(B.total_frames, 148), 256, 0, s>>>(B);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (with_grad && B.total_frames > 0) {
    batched_bwd_prologue<<<(unsigned)((B.total_frames + 127) / 128), 128, 0, s>>>(B);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (B.total_items > 0) {
      e = P.apt == 4 ? launch_stream<4, kBBwd>(B, P.grid_bwd, s) : launch_stream<8, kBBwd>(B, P.grid_bwd, s);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int batched_grid(int apt, bool backward, int sm_count, int64_t items) {
  const int occ = apt == 4 ? (backward ? occupancy_of<4, kBBwd>() : occupancy_of<4, kBFwd>())
                           : (backward ? occupancy_of<8, kBBwd>() : occupancy_of<8, kBFwd>());
  return (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * occ));
}

}  // namespace wmd

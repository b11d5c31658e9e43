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
#include <cstdlib>
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
  // the tile's 16-byte hull, then (gradient pass) the frame's 16-double rotation record
  static constexpr int kRecOffset = ((kTile * 3 * 4 + 32) + 127) / 128 * 128;
  static constexpr int kStageBytes = kRecOffset + kStatDoubles * 8;
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

// Copies item (t, f)'s coordinates into dst; with rot (the gradient pass) the
// frame's rotation record too, to dst + kRecOffset.
template <int APT>
__device__ __forceinline__ void batched_issue(const BatchSeg& s, int t, int64_t f, unsigned char* dst, uint64_t* bar,
                                              const double* rot) {
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
  mbar_arrive_expect_tx(bar, core + (rot ? (uint32_t)(kStatDoubles * 8) : 0u));
  if (core) bulk_copy_g2s(dst, base + c0, core, bar);
  if (rot) bulk_copy_g2s(dst + BGeo<APT>::kRecOffset, rot + (s.frame0 + f) * kStatDoubles, kStatDoubles * 8, bar);
}

template <int APT, int MODE>
__global__ void __launch_bounds__(kThreads, 4) batched_stream_kernel(const BatchLaunch B) {
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
  // the gradient pass stages each frame's rotation record with its coordinates
  const double* rec_src = MODE == kBBwd ? B.rot : nullptr;
  if (tid == 0) {
    cursor_init(B, w0, pc);
    for (; issued < S - 1 && issued < n_items; ++issued) {
      batched_issue<APT>(B.segs[pc.seg], pc.t, pc.f, smem + (issued % S) * G::kStageBytes, &full[issued % S], rec_src);
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
    // forward: refill at the top of the iteration; backward: after the
    // stage's gradient store has been issued (see below)
    if (MODE == kBFwd && tid == 0 && issued < n_items) {
      const int sp = (int)(issued % S);
      batched_issue<APT>(B.segs[pc.seg], pc.t, pc.f, smem + sp * G::kStageBytes, &full[sp], rec_src);
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
      // dRMSD/dx is written over x in the stage (each thread its own atoms),
      // then leaves by one bulk store of the tile's 16-byte-aligned middle and
      // at most 2 x 3 scalar floats at its ends.
      float* gs = const_cast<float*>(xs);
      const bool has_grad = sg.grad != nullptr;
      if (ok && has_grad) {
        const double* rt = reinterpret_cast<const double*>(smem + s * G::kStageBytes + G::kRecOffset);
        double R[9], cc[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) R[e] = rt[e];
        cc[0] = rt[9]; cc[1] = rt[10]; cc[2] = rt[11];
        const double scale = rt[12];
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          const int k = tid + j * kConsumerThreads;
          if (k < len) {
            const float x0 = gs[k * 3 + 0], x1 = gs[k * 3 + 1], x2 = gs[k * 3 + 2];
            const double ty0 = R[0] * yr[j][0] + R[3] * yr[j][1] + R[6] * yr[j][2];
            const double ty1 = R[1] * yr[j][0] + R[4] * yr[j][1] + R[7] * yr[j][2];
            const double ty2 = R[2] * yr[j][0] + R[5] * yr[j][1] + R[8] * yr[j][2];
            gs[k * 3 + 0] = (float)(scale * (((double)x0 - cc[0]) - ty0));
            gs[k * 3 + 1] = (float)(scale * (((double)x1 - cc[1]) - ty1));
            gs[k * 3 + 2] = (float)(scale * (((double)x2 - cc[2]) - ty2));
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      named_barrier_sync(1, kConsumerThreads);
      // byte range of this item in the gradient array and its aligned middle
      const uint64_t b0 = (uint64_t)(c.f * sg.n_atoms + a0) * 12ull;
      const uint64_t b1 = b0 + (uint64_t)len * 12ull;
      const uint64_t m0 = (b0 + 15ull) & ~15ull, m1 = b1 & ~15ull;
      const bool mid = m1 > m0;
      unsigned char* gbase = reinterpret_cast<unsigned char*>(sg.grad);
      const unsigned char* sbase = reinterpret_cast<const unsigned char*>(gs) - (b0 & 15ull);  // holds byte b0 & ~15
      if (tid == 0) {
        if (ok && has_grad && !*abort_flag && mid) {
          bulk_copy_s2g(gbase + m0, sbase + (m0 - (b0 & ~15ull)), (uint32_t)(m1 - m0));
        }
        bulk_commit();
        // the stage read by the previous item's store is refilled next
        bulk_wait_read<1>();
        if (issued < n_items) {
          const int sp = (int)(issued % S);
          batched_issue<APT>(B.segs[pc.seg], pc.t, pc.f, smem + sp * G::kStageBytes, &full[sp], rec_src);
          ++issued;
          cursor_next(B, pc);
        }
      } else if (ok && has_grad && tid >= 32 && tid < 38) {
        // ends outside the aligned middle: [b0, m0) and [m1, b1), or all of [b0, b1)
        const int q = tid - 32;  // 0..2 head, 3..5 tail
        const uint64_t at = mid ? (q < 3 ? b0 + 4ull * q : m1 + 4ull * (q - 3)) : b0 + 4ull * q;
        const uint64_t lim = mid ? (q < 3 ? m0 : b1) : b1;
        if (at < lim)
          *reinterpret_cast<float*>(gbase + at) = *reinterpret_cast<const float*>(sbase + (at - (b0 & ~15ull)));
      }
    } else {
      double acc[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[e] = 0.0;
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        if ((warp << 5) + j * kConsumerThreads >= len) break;  // warp-uniform: the rest of the tile is empty
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
    if (MODE == kBBwd) bulk_wait_all<0>();
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
  if (n == 0) {
    // empty selection: RMSD 0 for every frame
    for (int64_t f = tid; f < s.n_frames; f += blockDim.x) s.rmsd[f] = 0.0;
    return;
  }
  if (s.n_frames == 0) return;
  double m0 = 0, m1 = 0, m2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) { m0 += ref[k * 3]; m1 += ref[k * 3 + 1]; m2 += ref[k * 3 + 2]; }
  sum3(m0, m1, m2);
  const double inv = 1.0 / (double)n;
  m0 *= inv; m1 *= inv; m2 *= inv;
  if (tid == 0) { s.mean_y[0] = m0; s.mean_y[1] = m1; s.mean_y[2] = m2; }
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

// Frames of the batch, a lane each: the warp first sums the tile partials of
// its 32 frames in tile order (two frames at a time, 16 lanes per frame, into
// shared memory), then every lane runs QCP for its own frame -- the FP64
// Newton iteration and, with gradients, the rotation from the eigenvector --
// so the warp issues each instruction once for 32 frames.
__global__ void __launch_bounds__(256) batched_finalize(const BatchLaunch B) {
  __shared__ double st[8][32][17];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = ((int64_t)blockIdx.x * 8 + warp) * 32;
  if (base >= B.total_frames) return;
  for (int i = 0; i < 16; ++i) {
    const int fl = 2 * i + (lane >> 4);
    const int64_t g = base + fl;
    double v = 0.0;
    if (g < B.total_frames) {
      const BatchSeg& sg = B.segs[seg_of(B.segs, B.n_segs, g, true)];
      const int64_t f = g - sg.frame0;
      for (int t = 0; t < sg.n_tiles; ++t)
        v += B.partial[(size_t)(sg.item0 + (int64_t)t * sg.n_frames + f) * kStatDoubles + (lane & 15)];
    }
    st[warp][fl][lane & 15] = v;
  }
  __syncwarp();
  const int64_t g = base + lane;
  if (g >= B.total_frames) return;
  const BatchSeg& sg = B.segs[seg_of(B.segs, B.n_segs, g, true)];
  const int64_t f = g - sg.frame0;
  if (sg.n_atoms == 0) {
    // empty selection: RMSD 0, no rotation (the single-trajectory path writes the same)
    sg.rmsd[f] = 0.0;
    if (B.rot)
      for (int e = 0; e < 16; ++e) B.rot[g * kStatDoubles + e] = 0.0;
    return;
  }
  const double* tot = st[warp][lane];
  const double n = (double)sg.n_atoms, inv_n = 1.0 / n;
  const double sx[3] = {tot[0], tot[1], tot[2]};
  double h[9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) h[a * 3 + b] = tot[6 + a * 3 + b] - sx[a] * sg.sum_c[b] * inv_n;
  const double gx = tot[3] + tot[4] + tot[5] - (sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]) * inv_n;
  const QcpOut q = qcp_lambda(h, 0.5 * (gx + sg.gy));
  const double rmsd = sqrt(msd_from(gx, sg.gy, q.lambda, n));
  sg.rmsd[f] = rmsd;
  if (B.rot) {
    // per frame: R from the QCP eigenvector, centroid, 1 / (n rmsd)
    double r[9];
    rotation_from_qcp(h, q.lambda, r);
    double* o = B.rot + g * kStatDoubles;
    for (int e = 0; e < 9; ++e) o[e] = r[e];
    o[9] = sx[0] * inv_n; o[10] = sx[1] * inv_n; o[11] = sx[2] * inv_n;
    o[12] = rmsd > 0.0 ? 1.0 / (n * rmsd) : 0.0;
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
      if (B.rot) B.rot[g * kStatDoubles + 12] = rmsd > 0.0 ? 1.0 / ((double)sg.n_atoms * rmsd) : 0.0;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Frame-major fused kernel.  Frames are taken in groups: up to kGroupFrames
// consecutive frames of one trajectory holding at most kGroupBytes of
// coordinates (one frame when a frame is larger).  Each persistent CTA owns a
// contiguous run of groups of equal estimated cost.  Per group:
//   pass 1  the frames' 1-D chunks stream through the shared-memory ring; each
//           thread keeps its 15 FP64 sums of the current frame (sum x, sum x^2,
//           sum x y^T with the raw float reference y) in registers across the
//           frame's chunks; one reduction per frame;
//   finish  warp 0 runs QCP, the rotation and the near-zero residual check for
//           all frames of the group at once, one lane per frame (the residual
//           pass, when needed, re-reads the frame with plain loads);
//   pass 2  (gradients) the group's chunks stream again -- from L2, since the
//           group was read a few microseconds earlier -- and dRMSD/dx =
//           (x - xbar - R^T (y - ybar)) / (n RMSD) is written over x in the
//           stage and leaves by one bulk store per chunk.
// HBM traffic is 12 B per atom-frame read + 12 B written.  H = sum x y^T -
// (sum x) ybar^T loses nothing that matters in FP64: every product of two
// floats is exact and the correction is one rounding of a sum.

constexpr int kFrameConsts = 24;

template <int APT>
struct FGeo {
  using G = BGeo<APT>;
  static constexpr int kStatsOffset = G::kAbortOffset + 16;                         // [kGroupFrames][16]
  static constexpr int kConstOffset = kStatsOffset + kGroupFrames * 16 * 8;          // [kGroupFrames][24]
  static constexpr int kSmemBytes = kConstOffset + kGroupFrames * kFrameConsts * 8;
};

// global group whose start cost is the first at or after X
__device__ __forceinline__ int64_t group_at(const BatchLaunch& B, int64_t X) {
  int lo = 0, hi = B.n_segs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (B.segs[mid].cost0 <= X) lo = mid;
    else hi = mid - 1;
  }
  const BatchSeg& s = B.segs[lo];
  if (s.n_groups == 0) return s.group0;
  const int64_t gi = (X - s.cost0 + s.group_cost - 1) / s.group_cost;
  return s.group0 + (gi < s.n_groups ? gi : s.n_groups);
}

struct GroupCursor {
  int seg;
  int64_t gi;  // group index within the segment
  int pass;
  int j;       // frame within the group
  int t;       // chunk within the frame
};

__device__ __forceinline__ void group_seek(const BatchLaunch& B, int64_t grp, GroupCursor& c) {
  c.seg = 0;
  int lo = 0, hi = B.n_segs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (B.segs[mid].group0 <= grp) lo = mid;
    else hi = mid - 1;
  }
  c.seg = lo;
  c.gi = grp - B.segs[lo].group0;
  c.pass = 0;
  c.j = 0;
  c.t = 0;
}

__device__ __forceinline__ int group_count(const BatchSeg& s, int64_t gi) {
  const int64_t f0 = gi * s.m_group;
  const int64_t left = s.n_frames - f0;
  return (int)(left < s.m_group ? left : s.m_group);
}

template <int T, bool GRAD>
__device__ __forceinline__ void group_next_item(const BatchLaunch& B, GroupCursor& c) {
  const BatchSeg& s = B.segs[c.seg];
  const int nc = (int)((s.n_atoms + T - 1) / T);
  if (++c.t < nc) return;
  c.t = 0;
  if (++c.j < group_count(s, c.gi)) return;
  c.j = 0;
  if (GRAD && c.pass == 0 && s.grad != nullptr) {
    c.pass = 1;
    return;
  }
  c.pass = 0;
  if (++c.gi < s.n_groups) return;
  c.gi = 0;
  do {
    ++c.seg;
  } while (c.seg < B.n_segs && B.segs[c.seg].n_groups == 0);
}

// One lane: statistics -> RMSD, rotation and gradient constants.
// consts: [0..8] R (R (x - xbar) ~ y - ybar), [9..11] xbar - R^T ybar,
// [12] 1/(n rmsd), [13] rmsd, [14] residual pass needed, [16..18] xbar.
__device__ __noinline__ void frame_finish(const double* tot, const BatchSeg& sg, double* consts) {
  const double n = (double)sg.n_atoms, inv_n = 1.0 / n;
  const double sx[3] = {tot[0], tot[1], tot[2]};
  double h[9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) h[a * 3 + b] = tot[6 + a * 3 + b] - sx[a] * sg.mean_y[b];
  const double gx = tot[3] + tot[4] + tot[5] - (sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]) * inv_n;
  const QcpOut q = qcp_lambda(h, 0.5 * (gx + sg.gy));
  const double rmsd = sqrt(msd_from(gx, sg.gy, q.lambda, n));
  double r[9];
  rotation_from_qcp(h, q.lambda, r);
  const double xb[3] = {sx[0] * inv_n, sx[1] * inv_n, sx[2] * inv_n};
  for (int e = 0; e < 9; ++e) consts[e] = r[e];
  for (int i = 0; i < 3; ++i)
    consts[9 + i] = xb[i] - (r[0 * 3 + i] * sg.mean_y[0] + r[1 * 3 + i] * sg.mean_y[1] + r[2 * 3 + i] * sg.mean_y[2]);
  consts[12] = rmsd > 0.0 ? 1.0 / (n * rmsd) : 0.0;
  consts[13] = rmsd;
  consts[14] = rmsd < kRefineScale * (gx + sg.gy) * inv_n ? 1.0 : 0.0;
  consts[16] = xb[0]; consts[17] = xb[1]; consts[18] = xb[2];
}

template <int APT, bool GRAD>
__global__ void __launch_bounds__(kThreads, 4) batched_frame_kernel(const BatchLaunch B) {
  using G = BGeo<APT>;
  using FG = FGeo<APT>;
  constexpr int T = G::kTile;
  constexpr int S = G::kStages;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::kBarOffset);
  double* red = reinterpret_cast<double*>(smem + G::kRedOffset);   // [2][4 warps][16]
  double* stats = reinterpret_cast<double*>(smem + FG::kStatsOffset);
  double* consts = reinterpret_cast<double*>(smem + FG::kConstOffset);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::kAbortOffset);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t TC = B.total_cost;
  const int64_t G0 = blockIdx.x == 0 ? 0 : group_at(B, TC * (int64_t)blockIdx.x / gridDim.x);
  const int64_t G1 = blockIdx.x + 1 == gridDim.x ? B.total_groups
                                                 : group_at(B, TC * (int64_t)(blockIdx.x + 1) / gridDim.x);
  if (tid == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&full[st], 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (G1 <= G0) return;

  // producer (thread 0): walks the (group, pass, frame, chunk) items of [G0, G1)
  GroupCursor pc{0, 0, 0, 0, 0};
  int64_t issued = 0;
  auto producer_live = [&]() { return pc.seg < B.n_segs && B.segs[pc.seg].group0 + pc.gi < G1; };
  auto issue = [&]() {
    const int sp = (int)(issued % S);
    const BatchSeg& ps = B.segs[pc.seg];
    batched_issue<APT>(ps, pc.t, pc.gi * ps.m_group + pc.j, smem + sp * G::kStageBytes, &full[sp], nullptr);
    ++issued;
    group_next_item<T, GRAD>(B, pc);
  };
  if (tid == 0) {
    group_seek(B, G0, pc);
    while (issued < S - 1 && producer_live()) issue();
  }
  // end of every item: all consumers are done with the previous item's stage
  // and its gradient store (if any) has been read out, so it is refilled
  auto item_end = [&]() {
    if (tid == 0) {
      bulk_commit();
      bulk_wait_read<1>();
      if (producer_live()) issue();
    }
  };

  GroupCursor cc;
  group_seek(B, G0, cc);
  int s = 0;
  uint32_t phase = 0;
  int cache_seg = -1, cache_t = -1, pre_seg = -1, pre_t = -1;
  double yr[APT][3];
  float yn[APT][3];  // next chunk of the reference, loaded one item ahead
  bool stop = false;
  for (int64_t grp = G0; grp < G1 && !stop; ++grp) {
    while (cc.gi >= B.segs[cc.seg].n_groups) {  // segments without groups are never current
      cc.gi = 0;
      ++cc.seg;
    }
    const BatchSeg& sg = B.segs[cc.seg];
    const int64_t n = sg.n_atoms;
    const int nc = (int)((n + T - 1) / T);
    const int64_t f0 = cc.gi * sg.m_group;
    const int cnt = group_count(sg, cc.gi);
    auto fetch = [&](int t, float (&dst)[APT][3]) {
      const int64_t a0 = (int64_t)t * T;
      const int len = (int)(min(n, a0 + T) - a0);
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        const int k = tid + j * kConsumerThreads;
        if (k < len) {
          const float* y = sg.ref + (a0 + k) * 3;
          dst[j][0] = __ldg(y); dst[j][1] = __ldg(y + 1); dst[j][2] = __ldg(y + 2);
        } else {
          dst[j][0] = dst[j][1] = dst[j][2] = 0.f;
        }
      }
    };
    // reference chunk t into yr; for frames of several chunks the next
    // chunk's loads are issued now and land while this item is processed
    auto load_ref = [&](int t) {
      if (cc.seg != cache_seg || t != cache_t) {
        if (!(cc.seg == pre_seg && t == pre_t)) fetch(t, yn);
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          yr[j][0] = (double)yn[j][0]; yr[j][1] = (double)yn[j][1]; yr[j][2] = (double)yn[j][2];
        }
        cache_seg = cc.seg;
        cache_t = t;
      }
      if (nc > 1) {
        const int tn = t + 1 < nc ? t + 1 : 0;
        fetch(tn, yn);
        pre_seg = cc.seg;
        pre_t = tn;
      }
    };
    // ---- pass 1: statistics, one reduction per frame ----
    for (int j = 0; j < cnt && !stop; ++j) {
      const int64_t f = f0 + j;
      double acc[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[e] = 0.0;
      for (int t = 0; t < nc; ++t) {
        load_ref(t);
        const int64_t a0 = (int64_t)t * T;
        const int len = (int)(min(n, a0 + T) - a0);
        const bool ok = mbar_wait(&full[s], phase, B.status, kStatusTimeoutFull, abort_flag);
        const float* xs = reinterpret_cast<const float*>(smem + s * G::kStageBytes) +
                          (int)(((uint64_t)(f * n + a0) * 3) & 3ull);
#pragma unroll
        for (int q = 0; q < APT; ++q) {
          const int k = tid + q * kConsumerThreads;
          const bool in = ok && k < len;
          const double x0 = in ? (double)xs[k * 3 + 0] : 0.0;
          const double x1 = in ? (double)xs[k * 3 + 1] : 0.0;
          const double x2 = in ? (double)xs[k * 3 + 2] : 0.0;
          acc[0] += x0; acc[1] += x1; acc[2] += x2;
          acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
          acc[6] = fma(x0, yr[q][0], acc[6]);  acc[7] = fma(x0, yr[q][1], acc[7]);  acc[8] = fma(x0, yr[q][2], acc[8]);
          acc[9] = fma(x1, yr[q][0], acc[9]);  acc[10] = fma(x1, yr[q][1], acc[10]); acc[11] = fma(x1, yr[q][2], acc[11]);
          acc[12] = fma(x2, yr[q][0], acc[12]); acc[13] = fma(x2, yr[q][1], acc[13]); acc[14] = fma(x2, yr[q][2], acc[14]);
        }
        double* rb = red + (j & 1) * (kConsumerWarps * 16);
        if (t == nc - 1) {
          const double v = warp_reduce_scatter16(acc);
          if ((lane & 1) == 0) rb[warp * 16 + (lane >> 1)] = v;
        }
        named_barrier_sync(1, kConsumerThreads);
        if (t == nc - 1 && tid < 16)
          stats[j * 16 + tid] = rb[tid] + rb[16 + tid] + rb[32 + tid] + rb[48 + tid];
        item_end();
        if (++s == S) { s = 0; phase ^= 1u; }
        if (*abort_flag) { stop = true; break; }
      }
    }
    if (stop) break;
    // ---- finish: QCP for the whole group, one lane per frame ----
    named_barrier_sync(1, kConsumerThreads);
    if (warp == 0 && lane < cnt) {
      double* cj = consts + lane * kFrameConsts;
      frame_finish(stats + lane * 16, sg, cj);
      if (cj[14] == 0.0) sg.rmsd[f0 + lane] = cj[13];
    }
    named_barrier_sync(1, kConsumerThreads);
    for (int j = 0; j < cnt; ++j) {
      double* cj = consts + j * kFrameConsts;
      if (cj[14] == 0.0) continue;
      // near-zero RMSD: explicit residual |R (x - xbar) - (y - ybar)|^2 in FP64
      double R[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) R[e] = cj[e];
      const double xb0 = cj[16], xb1 = cj[17], xb2 = cj[18];
      const double yb0 = sg.mean_y[0], yb1 = sg.mean_y[1], yb2 = sg.mean_y[2];
      const float* frame = sg.coords + (size_t)(f0 + j) * n * 3;
      double r2 = 0.0;
      for (int64_t k = tid; k < n; k += kConsumerThreads) {
        const double d0 = (double)frame[k * 3] - xb0, d1 = (double)frame[k * 3 + 1] - xb1,
                     d2 = (double)frame[k * 3 + 2] - xb2;
        const double e0 = R[0] * d0 + R[1] * d1 + R[2] * d2 - ((double)sg.ref[k * 3] - yb0);
        const double e1 = R[3] * d0 + R[4] * d1 + R[5] * d2 - ((double)sg.ref[k * 3 + 1] - yb1);
        const double e2 = R[6] * d0 + R[7] * d1 + R[8] * d2 - ((double)sg.ref[k * 3 + 2] - yb2);
        r2 += e0 * e0 + e1 * e1 + e2 * e2;
      }
      for (int o = 16; o; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
      if (lane == 0) red[warp] = r2;
      named_barrier_sync(1, kConsumerThreads);
      if (tid == 0) {
        const double rmsd = sqrt((red[0] + red[1] + red[2] + red[3]) / (double)n);
        cj[13] = rmsd;
        cj[12] = rmsd > 0.0 ? 1.0 / ((double)n * rmsd) : 0.0;
        cj[14] = 0.0;
        sg.rmsd[f0 + j] = rmsd;
      }
      named_barrier_sync(1, kConsumerThreads);
    }
    // ---- pass 2: gradients ----
    if (GRAD && sg.grad != nullptr) {
      unsigned char* gbase = reinterpret_cast<unsigned char*>(sg.grad);
      for (int j = 0; j < cnt && !stop; ++j) {
        const int64_t f = f0 + j;
        const double* cj = consts + j * kFrameConsts;
        double R[9], dd[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) R[e] = cj[e];
        dd[0] = cj[9]; dd[1] = cj[10]; dd[2] = cj[11];
        const double scale = cj[12];
        for (int t = 0; t < nc; ++t) {
          load_ref(t);
          const int64_t a0 = (int64_t)t * T;
          const int len = (int)(min(n, a0 + T) - a0);
          const bool ok = mbar_wait(&full[s], phase, B.status, kStatusTimeoutFull, abort_flag);
          float* gs = reinterpret_cast<float*>(smem + s * G::kStageBytes) + (int)(((uint64_t)(f * n + a0) * 3) & 3ull);
          if (ok) {
#pragma unroll
            for (int q = 0; q < APT; ++q) {
              const int k = tid + q * kConsumerThreads;
              if (k < len) {
                const double x0 = gs[k * 3 + 0], x1 = gs[k * 3 + 1], x2 = gs[k * 3 + 2];
                const double ty0 = R[0] * yr[q][0] + R[3] * yr[q][1] + R[6] * yr[q][2];
                const double ty1 = R[1] * yr[q][0] + R[4] * yr[q][1] + R[7] * yr[q][2];
                const double ty2 = R[2] * yr[q][0] + R[5] * yr[q][1] + R[8] * yr[q][2];
                gs[k * 3 + 0] = (float)(scale * ((x0 - ty0) - dd[0]));
                gs[k * 3 + 1] = (float)(scale * ((x1 - ty1) - dd[1]));
                gs[k * 3 + 2] = (float)(scale * ((x2 - ty2) - dd[2]));
              }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          }
          named_barrier_sync(1, kConsumerThreads);
          const uint64_t b0 = (uint64_t)(f * n + a0) * 12ull;
          const uint64_t b1 = b0 + (uint64_t)len * 12ull;
          const uint64_t m0 = (b0 + 15ull) & ~15ull, m1 = b1 & ~15ull;
          const bool mid = m1 > m0;
          const unsigned char* sbase = reinterpret_cast<const unsigned char*>(gs) - (b0 & 15ull);
          if (tid == 0) {
            if (ok && !*abort_flag && mid)
              bulk_copy_s2g(gbase + m0, sbase + (m0 - (b0 & ~15ull)), (uint32_t)(m1 - m0));
          } else if (ok && tid >= 32 && tid < 38) {
            const int q = tid - 32;
            const uint64_t at = mid ? (q < 3 ? b0 + 4ull * q : m1 + 4ull * (q - 3)) : b0 + 4ull * q;
            const uint64_t lim = mid ? (q < 3 ? m0 : b1) : b1;
            if (at < lim)
              *reinterpret_cast<float*>(gbase + at) = *reinterpret_cast<const float*>(sbase + (at - (b0 & ~15ull)));
          }
          item_end();
          if (++s == S) { s = 0; phase ^= 1u; }
          if (*abort_flag) { stop = true; break; }
        }
      }
    }
    ++cc.gi;
  }
  if (tid == 0) {
    bulk_wait_all<0>();
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

// ---------------------------------------------------------------------------
// Lanes layout forward: units (trajectory, atom tile, 32-frame group); lane l
// of a warp accumulates frame 32g + l over the tile, in FP64 and in atom
// order, and stores the item partial (tile, frame) the finisher reads.  A
// stage is 32 atoms of the group's 32 frames plus the 32 reference atoms
// (FP64, centred; a 1-D bulk copy by lane 0), and its barrier counts 32
// arrivals.  The frames arrive by the trajectory's 2-D tensor map
// (batched_encode_maps), lane 0 issuing every box:
//   frame rows (tma = 1): 3 boxes of [32 frames x 32 floats], 128-byte
//       swizzle, so that the 32 lanes reading their own rows hit distinct
//       bank groups -- the layout of the single-trajectory lanes kernel;
//   quad rows (tma = 2): 4 boxes of [8 quad rows x 100 floats], box j holding
//       frame position j of quad rows 8g .. 8g + 7 from the 16-byte boundary
//       at or below the stage's first atom; lane 4i + j reads row i of box j
//       at a fixed float offset.  Lanes of the last n_frames mod 4 frames
//       (past the last whole quad row) read their atoms with plain loads.
// Without a map (tma = 0) every lane bulk-copies its own frame's row, the
// 16-byte hull of 32 atoms (at most 400 bytes).  Warps take contiguous runs
// of units of equal estimated cost.
// ---------------------------------------------------------------------------
constexpr int kBLWarps = 4;
constexpr int kBLStages = 2;
constexpr int kBLRow = 400;                // bytes per frame row of a per-lane stage
constexpr int kBLXBytes = 32 * kBLRow;     // 12,800: per-lane rows, or 4 quad boxes; 3 swizzled boxes take 12,288
constexpr int kBLQuadBox = 8 * kBLRow;     // [8 quad rows x 100 floats]
constexpr int kBLXStage = 13312;           // a frame slot, a multiple of 1024 bytes (128-byte swizzle)
constexpr int kBLYBytes = 32 * 3 * 8;
constexpr int kBLYOffset = kBLWarps * kBLStages * kBLXStage;
constexpr int kBLBarOffset = kBLYOffset + kBLWarps * kBLStages * kBLYBytes;
constexpr int kBLAbortOffset = kBLBarOffset + kBLWarps * kBLStages * 8;
constexpr int kBLSmemBytes = kBLAbortOffset + 16 + 1024;  // + slack to align the base to 1024
static_assert(kBLXBytes <= kBLXStage && 3 * 4096 <= kBLXStage && 4 * kBLQuadBox <= kBLXStage, "frame slot");

__device__ __forceinline__ void bl_tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// last segment whose units start at or before cost c
__device__ __forceinline__ int lane_seg_of(const BatchSeg* segs, int n, int64_t c) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].lane_cost0 <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct LaneCur {
  int seg;
  int64_t k;  // unit within the segment
};

// The fields of a trajectory the lanes kernel reads per stage and per unit,
// held in registers while a cursor stays in that trajectory.
struct LaneSeg {
  const float* coords;
  const double* yc;
  int64_t n_atoms, n_frames, groups, item0;
  int64_t cost0, full_units, unit_cost, last_cost;
  int tma;
};

__device__ __forceinline__ LaneSeg lane_seg(const BatchSeg& S) {
  LaneSeg v;
  v.coords = S.coords;
  v.yc = S.yc;
  v.n_atoms = S.n_atoms;
  v.n_frames = S.n_frames;
  v.groups = (S.n_frames + 31) / 32;
  v.item0 = S.item0;
  v.cost0 = S.lane_cost0;
  v.full_units = S.lane_full_units;
  v.unit_cost = S.lane_unit_cost;
  v.last_cost = S.lane_last_cost;
  v.tma = S.tma;
  return v;
}

// a unit's starting cost: whole-tile units first, then the last tile's
__device__ __forceinline__ int64_t lane_unit_start(const LaneSeg& v, int64_t k) {
  return v.cost0 + (k <= v.full_units ? k * v.unit_cost : v.full_units * v.unit_cost + (k - v.full_units) * v.last_cost);
}

__device__ __forceinline__ void lane_skip_empty(const BatchLaunch& B, LaneCur& c) {
  while (c.seg < B.n_segs && c.k >= B.segs[c.seg].lane_units) {
    ++c.seg;
    c.k = 0;
  }
}

template <int APT>
__global__ void __launch_bounds__(kBLWarps * 32) batched_lanes_kernel(const BatchLaunch B) {
  constexpr int T = kConsumerThreads * APT;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBLBarOffset);
  uint64_t* full = bars + warp * kBLStages;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + kBLAbortOffset);
  unsigned char* ring = smem + warp * kBLStages * kBLXStage;
  unsigned char* yring = smem + kBLYOffset + warp * kBLStages * kBLYBytes;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kBLWarps * kBLStages; ++i) mbar_init(&bars[i], 32);
    *abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t nw = (int64_t)gridDim.x * kBLWarps, gw = (int64_t)blockIdx.x * kBLWarps + warp;
  const int64_t C0 = B.total_lane_cost * gw / nw, C1 = B.total_lane_cost * (gw + 1) / nw;
  if (C0 >= C1 || B.n_segs == 0) return;
  // first unit starting at or after C0
  LaneCur first;
  first.seg = lane_seg_of(B.segs, B.n_segs, C0);
  {
    const BatchSeg& S = B.segs[first.seg];
    const int64_t off = C0 - S.lane_cost0;
    const int64_t full = S.lane_full_units * S.lane_unit_cost;
    if (S.lane_units <= 0) first.k = 0;
    else if (off <= full) first.k = (off + S.lane_unit_cost - 1) / S.lane_unit_cost;
    else first.k = S.lane_full_units + (off - full + S.lane_last_cost - 1) / S.lane_last_cost;
  }
  lane_skip_empty(B, first);
  // a cursor's trajectory view, reloaded when the cursor enters another trajectory
  auto view = [&](const LaneCur& c, int& vseg, LaneSeg& v) {
    if (c.seg < B.n_segs && c.seg != vseg) {
      v = lane_seg(B.segs[c.seg]);
      vseg = c.seg;
    }
  };
  auto starts_before_end = [&](const LaneCur& c, const LaneSeg& v) {
    return c.seg < B.n_segs && lane_unit_start(v, c.k) < C1;
  };
  auto unit_stages = [&](const LaneCur& c, const LaneSeg& v) {
    const int64_t t = c.k / v.groups;
    return (int)((min((int64_t)T, v.n_atoms - t * T) + 31) / 32);
  };
  // producer cursor: unit pc (tile pt, frame group pg), stage pj; every lane runs it (warp-uniform)
  LaneCur pc = first;
  int pv_seg = -1;
  LaneSeg pv;
  view(pc, pv_seg, pv);
  int pj = 0;
  bool p_live = starts_before_end(pc, pv);
  int p_st = p_live ? unit_stages(pc, pv) : 0;
  int64_t pt = p_live ? pc.k / pv.groups : 0, pg = p_live ? pc.k - pt * pv.groups : 0;
  int64_t n_issued = 0;
  auto issue_next = [&]() {
    const int64_t t = pt, g = pg;
    const int64_t a0 = t * T + (int64_t)pj * 32;
    const int nv = (int)min((int64_t)32, pv.n_atoms - a0);
    const int slot = (int)(n_issued % kBLStages);
    unsigned char* st = ring + slot * kBLXStage;
    unsigned char* ys = yring + slot * kBLYBytes;
    unsigned char* dst = st + lane * kBLRow;
    const int64_t f = g * 32 + lane;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (pv.tma) {
      if (lane == 0) {
        const CUtensorMap* map = B.maps + pc.seg;
        mbar_arrive_expect_tx(&full[slot], (pv.tma == 1 ? 3 * 4096 : 4 * kBLQuadBox) + kBLYBytes);
        if (pv.tma == 1) {
#pragma unroll
          for (int b = 0; b < 3; ++b) bl_tma_load_2d(st + b * 4096, map, (int)(a0 * 3 + 32 * b), (int)(g * 32), &full[slot]);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int64_t e = (int64_t)j * 3 * pv.n_atoms + 3 * a0;
            bl_tma_load_2d(st + j * kBLQuadBox, map, (int)(e & ~int64_t(3)), (int)(g * 8), &full[slot]);
          }
        }
        bulk_copy_g2s(ys, pv.yc + a0 * 3, kBLYBytes, &full[slot]);
      } else {
        mbar_arrive(&full[slot]);
      }
    } else {
      uint32_t bytes = 0;
      uint64_t c0 = 0;
      const unsigned char* base = reinterpret_cast<const unsigned char*>(pv.coords);
      if (f < pv.n_frames) {
        const uint64_t total_al = ((uint64_t)pv.n_frames * (uint64_t)pv.n_atoms * 12ull) & ~15ull;
        const uint64_t b0 = (uint64_t)(f * pv.n_atoms + a0) * 12ull;
        const uint64_t b1 = b0 + (uint64_t)nv * 12ull;
        c0 = b0 & ~15ull;
        uint64_t c1 = (b1 + 15ull) & ~15ull;
        if (c1 > total_al) {  // the array's unaligned tail: plain loads
          const uint64_t tail0 = total_al > c0 ? total_al : c0;
          for (uint64_t bb = tail0; bb < b1; bb += 4)
            *reinterpret_cast<float*>(dst + (bb - c0)) = __ldg(reinterpret_cast<const float*>(base + bb));
          c1 = tail0;
        }
        bytes = (uint32_t)(c1 - c0);
      }
      const uint32_t tx = bytes + (lane == 0 ? (uint32_t)kBLYBytes : 0u);
      if (tx) mbar_arrive_expect_tx(&full[slot], tx);
      else mbar_arrive(&full[slot]);
      if (bytes) bulk_copy_g2s(dst, base + c0, bytes, &full[slot]);
      if (lane == 0) bulk_copy_g2s(ys, pv.yc + a0 * 3, kBLYBytes, &full[slot]);
    }
    ++n_issued;
    if (++pj == p_st) {
      pj = 0;
      ++pc.k;
      lane_skip_empty(B, pc);
      view(pc, pv_seg, pv);
      p_live = starts_before_end(pc, pv);
      if (p_live) {
        p_st = unit_stages(pc, pv);
        pt = pc.k / pv.groups;
        pg = pc.k - pt * pv.groups;
      } else {
        p_st = 0;
      }
    }
  };
  while (p_live && n_issued < kBLStages) issue_next();

  int64_t n_done = 0;
  bool aborted = false;
  LaneCur cu = first;
  int cv_seg = -1;
  LaneSeg cv;
  view(cu, cv_seg, cv);
  while (starts_before_end(cu, cv) && !aborted) {
    const LaneSeg& S = cv;
    const int64_t groups = S.groups;
    const int64_t t = cu.k / groups, g = cu.k - t * groups;
    const int st_n = unit_stages(cu, cv);
    const int64_t f = g * 32 + lane;
    const bool live = f < S.n_frames;
    // quad rows: this lane's float offset into its box row; lanes past the
    // last whole quad row read from global memory
    const int quad_off = (int)(((int64_t)(lane & 3) * 3 * S.n_atoms) & 3);
    const bool quad_tail = S.tma == 2 && f >= (S.n_frames & ~int64_t(3));
    double acc[15];
#pragma unroll
    for (int e = 0; e < 15; ++e) acc[e] = 0.0;
    for (int j = 0; j < st_n; ++j) {
      const int slot = (int)(n_done % kBLStages);
      const uint32_t parity = (uint32_t)((n_done / kBLStages) & 1);
      if (!mbar_wait(&full[slot], parity, B.status, kStatusTimeoutFull, abort_flag)) {
        aborted = true;
        break;
      }
      const int64_t a0 = t * T + (int64_t)j * 32;
      const int nv = (int)min((int64_t)32, S.n_atoms - a0);
      const unsigned char* st = ring + slot * kBLXStage;
      const double* ys = reinterpret_cast<const double*>(yring + slot * kBLYBytes);
      auto add = [&](double x0, double x1, double x2, int a) {
        const double y0 = ys[3 * a], y1 = ys[3 * a + 1], y2 = ys[3 * a + 2];
        acc[0] += x0; acc[1] += x1; acc[2] += x2;
        acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
        acc[6] = fma(x0, y0, acc[6]);  acc[7] = fma(x0, y1, acc[7]);  acc[8] = fma(x0, y2, acc[8]);
        acc[9] = fma(x1, y0, acc[9]);  acc[10] = fma(x1, y1, acc[10]); acc[11] = fma(x1, y2, acc[11]);
        acc[12] = fma(x2, y0, acc[12]); acc[13] = fma(x2, y1, acc[13]); acc[14] = fma(x2, y2, acc[14]);
      };
      if (live && S.tma == 1) {
        // 4 atoms = 3 swizzled 16-byte chunks of this lane's 128-byte row in each box
        const unsigned char* row = st + lane * 128;
        const int sw = lane & 7;
        auto chunk = [&](int c) -> float4 {
          return *reinterpret_cast<const float4*>(row + (c >> 3) * 4096 + (((c & 7) ^ sw) << 4));
        };
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          if (4 * m >= nv) break;
          const float4 p = chunk(3 * m), q = chunk(3 * m + 1), r = chunk(3 * m + 2);
          add(p.x, p.y, p.z, 4 * m);
          if (4 * m + 1 < nv) add(p.w, q.x, q.y, 4 * m + 1);
          if (4 * m + 2 < nv) add(q.z, q.w, r.x, 4 * m + 2);
          if (4 * m + 3 < nv) add(r.y, r.z, r.w, 4 * m + 3);
        }
      } else if (live) {
        const float* xr;
        if (S.tma == 2 && !quad_tail) {
          xr = reinterpret_cast<const float*>(st + (lane & 3) * kBLQuadBox + (lane >> 2) * kBLRow) + quad_off;
        } else if (S.tma == 2) {
          xr = S.coords + ((size_t)f * S.n_atoms + a0) * 3;
        } else {
          const int head = (int)(((uint64_t)(f * S.n_atoms + a0) * 12ull) & 15ull);
          xr = reinterpret_cast<const float*>(st + lane * kBLRow + head);
        }
#pragma unroll 4
        for (int a = 0; a < nv; ++a) add(xr[3 * a], xr[3 * a + 1], xr[3 * a + 2], a);
      }
      ++n_done;
      __syncwarp();
      if (p_live) issue_next();
    }
    if (aborted) break;
    if (live) {
      double2* rec = reinterpret_cast<double2*>(B.partial + (size_t)(S.item0 + t * S.n_frames + f) * kStatDoubles);
#pragma unroll
      for (int e = 0; e < 7; ++e) rec[e] = make_double2(acc[2 * e], acc[2 * e + 1]);
      rec[7] = make_double2(acc[14], 0.0);
    }
    ++cu.k;
    lane_skip_empty(B, cu);
    view(cu, cv_seg, cv);
  }
  // after an abort, copies this warp issued may still be landing
  if (aborted) {
    for (int64_t j = n_done; j < n_issued; ++j) {
      const int slot = (int)(j % kBLStages);
      const uint32_t ph = (uint32_t)((j / kBLStages) & 1);
      const uint64_t t0 = global_timer_ns();
      while (!mbar_try_wait(&full[slot], ph)) {
        if (global_timer_ns() - t0 > kWaitLimitNs) {
          atomicOr(B.status, kStatusTimeoutDrain);
          break;
        }
      }
    }
  }
}

template <int APT>
cudaError_t launch_lanes(const BatchLaunch& B, int grid, cudaStream_t s) {
  auto kern = batched_lanes_kernel<APT>;
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kBLSmemBytes);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  kern<<<grid, kBLWarps * 32, kBLSmemBytes, s>>>(B);
  return cudaGetLastError();
}

template <int APT, bool GRAD>
cudaError_t launch_frames(const BatchLaunch& B, int grid, cudaStream_t s) {
  auto kern = batched_frame_kernel<APT, GRAD>;
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, FGeo<APT>::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  kern<<<grid, kThreads, FGeo<APT>::kSmemBytes, s>>>(B);
  return cudaGetLastError();
}

template <int APT, bool GRAD>
int frame_occupancy() {
  auto kern = batched_frame_kernel<APT, GRAD>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, FGeo<APT>::kSmemBytes);
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kThreads, FGeo<APT>::kSmemBytes) != cudaSuccess)
    blocks = 1;
  return blocks < 1 ? 1 : blocks;
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

bool batched_encode_maps(std::vector<BatchSeg>& segs, CUtensorMap* maps, std::string* msg) {
  using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeTiled enc = nullptr;
  const char* env = std::getenv("WARPMD_BATCHED_TMA");
  const bool off = env && std::strcmp(env, "0") == 0;
  for (BatchSeg& g : segs) g.tma = 0;
  if (off) return true;
  if (!enc) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p) {
      cudaGetLastError();
      *msg = "cuda driver error: cuTensorMapEncodeTiled unavailable";
      return false;
    }
    enc = reinterpret_cast<EncodeTiled>(p);
  }
  for (size_t i = 0; i < segs.size(); ++i) {
    BatchSeg& g = segs[i];
    std::memset(&maps[i], 0, sizeof(CUtensorMap));
    const int64_t n = g.n_atoms, F = g.n_frames;
    if (n <= 0 || F < 4 || !g.coords) continue;
    const bool rows = n % 4 == 0;
    const cuuint64_t dims[2] = {(cuuint64_t)(rows ? 3 * n : 12 * n), (cuuint64_t)(rows ? F : F / 4)};
    const cuuint64_t stride[1] = {(cuuint64_t)(rows ? 12 * n : 48 * n)};
    const cuuint32_t box[2] = {rows ? 32u : 100u, rows ? 32u : 8u};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(g.coords), dims, stride, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           rows ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      *msg = "cuda driver error: tensor map of batched trajectory " + std::to_string(i) + " (CUresult " +
             std::to_string((int)r) + ", " + std::to_string((long long)n) + " atoms, " + std::to_string((long long)F) +
             " frames)";
      return false;
    }
    g.tma = rows ? 1 : 2;
  }
  return true;
}

int batched_tile_atoms(int apt) { return kConsumerThreads * apt; }

cudaError_t batched_enqueue(const BatchPlan& P, bool with_grad, cudaStream_t s) {
  BatchLaunch B = P.launch;
  cudaError_t e;
  batched_ref_prep<<<P.n_segs, 256, 0, s>>>(P.segs_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (P.variant == kBatchFrames) {
    if (B.total_groups == 0) return cudaSuccess;
    if (P.apt == 4)
      return with_grad ? launch_frames<4, true>(B, P.grid_fwd, s) : launch_frames<4, false>(B, P.grid_fwd, s);
    return with_grad ? launch_frames<8, true>(B, P.grid_fwd, s) : launch_frames<8, false>(B, P.grid_fwd, s);
  }
  if ((e = cudaMemsetAsync(B.refine_count, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
  if (B.total_items > 0) {
    if (P.variant == kBatchLanes)
      e = P.apt == 4 ? launch_lanes<4>(B, P.grid_fwd, s) : launch_lanes<8>(B, P.grid_fwd, s);
    else
      e = P.apt == 4 ? launch_stream<4, kBFwd>(B, P.grid_fwd, s) : launch_stream<8, kBFwd>(B, P.grid_fwd, s);
    if (e != cudaSuccess) return e;
  }
  if (B.total_frames > 0) {
    batched_finalize<<<(unsigned)((B.total_frames + 255) / 256), 256, 0, s>>>(B);
    batched_refine<<<(unsigned)std::min<int64_t>(B.total_frames, 148), 256, 0, s>>>(B);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (with_grad && B.total_items > 0) {
    e = P.apt == 4 ? launch_stream<4, kBBwd>(B, P.grid_bwd, s) : launch_stream<8, kBBwd>(B, P.grid_bwd, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int batched_grid(int apt, bool backward, int sm_count, int64_t items) {
  const int occ = apt == 4 ? (backward ? occupancy_of<4, kBBwd>() : occupancy_of<4, kBFwd>())
                           : (backward ? occupancy_of<8, kBBwd>() : occupancy_of<8, kBFwd>());
  return (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * occ));
}

int batched_lanes_grid(int sm_count, int64_t units) {
  static int occ = 0;
  if (occ == 0) {
    cudaFuncSetAttribute(batched_lanes_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBLSmemBytes);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batched_lanes_kernel<8>, kBLWarps * 32, kBLSmemBytes) !=
        cudaSuccess)
      b = 1;
    occ = std::max(b, 1);
  }
  const int64_t by_units = (units + kBLWarps - 1) / kBLWarps;
  return (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count * occ, by_units));
}

int batched_frame_grid(int apt, bool with_grad, int sm_count, int64_t groups) {
  const int occ = apt == 4 ? (with_grad ? frame_occupancy<4, true>() : frame_occupancy<4, false>())
                           : (with_grad ? frame_occupancy<8, true>() : frame_occupancy<8, false>());
  return (int)std::max<int64_t>(1, std::min<int64_t>(groups, (int64_t)sm_count * occ));
}

}  // namespace wmd

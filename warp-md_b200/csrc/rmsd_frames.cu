// rmsd_frames.cu -- per-frame RMSD (forward) and dRMSD/dx (backward) kernels.
//
// Replaces the reference's rmsd_centroid / rmsd_cov / rmsd_raw_accum /
// rmsd_finalize NVRTC kernels (crates/traj-kernels/src/kernels/part1.cu:299-393)
// and the host-side rmsd_from_cov SVD (crates/traj-engine/src/plans/rmsd/math.rs:7-38)
// with one fused, persistent launch:
//
//   * Work items are (atom tile, frame) pairs, tile-major; each CTA owns a
//     contiguous, balanced run of items.  Frames are float32 coordinates,
//     frame-major [frame][atom][stride].
//   * A producer warp streams each item's contiguous byte range into a ring of
//     shared-memory stages with 1-D bulk async copies (cp.async.bulk, TMA
//     without a tensor map, no multicast) completing on mbarriers.  The 16-byte
//     aligned hull of the range is copied; the consumers index past the head
//     remainder.  Only the last item of the array can end in an unaligned tail,
//     which the producer fills with plain loads.
//   * 8 consumer warps hold the item's reference atoms in registers (centred,
//     FP64) and accumulate per frame, in FP64, sum x (3), sum x_a^2 (3) and
//     P = sum x y_c^T (9) -- all statistics the QCP needs in one pass.  Frames
//     are not pre-centred: with y_c centred, H = P - x_bar (sum y_c)^T exactly.
//   * The 15 sums are reduced across the CTA with a butterfly reduce-scatter
//     (16 shuffles) and a 2 KB shared buffer, and stored as a 16-double
//     partial per (frame, tile).  A finalize kernel adds each frame's partials
//     in tile order -- so results are bitwise reproducible -- and runs QCP in
//     FP64; the streaming loop itself never fences or waits on other CTAs.
//   * Bounded waits everywhere: a wait that exceeds kWaitLimitNs records a
//     status bit in the context's status word and the CTA exits after letting
//     its copies in flight land.
//
// The backward kernel streams the same items again, re-derives R from the QCP
// eigenvector of the stored H (a per-frame prologue kernel), and writes
// grad = dL/drmsd * (x - x_bar - R^T y_c) / (n rmsd) as float32.
//
// Gathered forward launches (atoms by index, or an unaligned base) run
// rmsd_gather_kernel instead: a warp per item, no staging, the same partials.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_util.cuh"
#include "qcp.cuh"
#include "wmd_internal.h"

namespace wmd {

enum Mode : int { kFwdFit = 0, kFwdRaw = 1, kBwd = 2, kFwdW = 3 };

template <int STRIDE, int APT>
struct Geo {
  static constexpr int kTile = kConsumerThreads * APT;
  // the tile's 16-byte hull, then (gradient pass) the frame's 16-double rotation record
  static constexpr int kRecOffset = ((kTile * STRIDE * 4 + 32) + 127) / 128 * 128;
  static constexpr int kStageBytes = kRecOffset + kStatDoubles * 8;
  static constexpr int kStagesRaw = 51200 / kStageBytes;
  static constexpr int kStages = kStagesRaw < 3 ? 3 : (kStagesRaw > 8 ? 8 : kStagesRaw);
  static constexpr int kRedBytes = 2 * kConsumerWarps * 16 * 8;
  static constexpr int kBarOffset = kStages * kStageBytes;
  static constexpr int kRedOffset = kBarOffset + kStages * 8;
  static constexpr int kAbortOffset = kRedOffset + kRedBytes;
  static constexpr int kSmemBytes = kAbortOffset + 16;
};

// Everything a finished frame needs: the 15 CTA/partial sums in lanes 0..14.
__device__ __noinline__ void finish_frame(const FrameLaunch& L, int64_t f, double v, int mode) {
  double tot[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) tot[e] = __shfl_sync(0xffffffffu, v, e);
  if ((threadIdx.x & 31) != 0) return;
  const double n = (double)L.ref.n_sel;
  if (mode == kFwdRaw) {
    // tot[0] = sum |x - y|^2 accumulated directly
    const double msd = n > 0 ? tot[0] / n : 0.0;
    if (L.out.rmsd) L.out.rmsd[f] = sqrt(msd);
    return;
  }
  const double inv_n = 1.0 / n;
  const double sx[3] = {tot[0], tot[1], tot[2]};
  const double sxx = tot[3] + tot[4] + tot[5];
  double h[9];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) h[a * 3 + b] = tot[6 + a * 3 + b] - sx[a] * L.ref.sum_c[b] * inv_n;
  const double gx = sxx - (sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]) * inv_n;
  const double gy = L.ref.gy;
  const QcpOut q = qcp_lambda(h, 0.5 * (gx + gy));
  const double rmsd = sqrt(msd_from(gx, gy, q.lambda, n));
  if (L.out.rmsd) L.out.rmsd[f] = rmsd;
  if (L.refine && (L.out.rmsd || L.out.stats) && rmsd < kRefineScale * (gx + gy) * inv_n) {
    // near-zero RMSD: queue the frame for the explicit residual pass
    const unsigned slot = atomicAdd(L.refine_count, 1u);
    double* rec = L.refine + (size_t)slot * kStatDoubles;
    rec[0] = (double)f;
    rec[1] = sx[0] * inv_n; rec[2] = sx[1] * inv_n; rec[3] = sx[2] * inv_n;
#pragma unroll
    for (int e = 0; e < 9; ++e) rec[4 + e] = h[e];
    rec[13] = q.lambda;
  }
  if (L.out.stats) {
    double* st = L.out.stats + f * kStatDoubles;
    st[0] = sx[0] * inv_n; st[1] = sx[1] * inv_n; st[2] = sx[2] * inv_n;
#pragma unroll
    for (int e = 0; e < 9; ++e) st[3 + e] = h[e];
    st[12] = q.lambda; st[13] = rmsd; st[14] = n; st[15] = gx + gy;
  }
  if (L.out.cov) {
#pragma unroll
    for (int e = 0; e < 9; ++e) L.out.cov[f * 9 + e] = (float)h[e];
  }
  if (L.out.sum_x2) L.out.sum_x2[f] = (float)gx;
  if (L.out.sum_y2) L.out.sum_y2[f] = (float)gy;
}

// Leader warp of an item: total over the 8 consumer warps, stored as the
// item's 16-double partial.  No fence and no atomic here: frames are finished
// by rmsd_finalize_kernel after the streaming kernel has ended.
__device__ __forceinline__ void item_epilogue(const FrameLaunch& L, const double* red, int n_tiles, int t,
                                              int64_t f) {
  const int lane = threadIdx.x & 31;
  if (lane < 16) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kConsumerWarps; ++w) v += red[w * 16 + lane];
    L.partial[((size_t)f * n_tiles + t) * kStatDoubles + lane] = v;
  }
}

// One warp per frame: adds the frame's tile partials in tile order (so results
// are bitwise reproducible), then QCP / outputs in finish_frame.
template <int MODE>
__global__ void __launch_bounds__(256) rmsd_finalize_kernel(const FrameLaunch L, int n_tiles) {
  const int64_t f = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (f >= L.n_frames) return;
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  if (lane < 16) {
    const double* part = L.partial + (size_t)f * n_tiles * kStatDoubles + lane;
    for (int tt = 0; tt < n_tiles; ++tt) s += part[(size_t)tt * kStatDoubles];
  }
  finish_frame(L, f, s, MODE);
}

// Byte range of item (t, f) and its bulk copy into a stage.  The 16-byte
// aligned hull [c0, c1) is copied; a range that runs into the unaligned tail
// of the array gets its last floats by plain loads.  With rec_offset > 0 (the
// gradient pass) frame f's rotation record follows at dst + rec_offset.
// Called by one thread.
template <int STRIDE, int T>
__device__ __forceinline__ void issue_item(const FrameLaunch& L, int t, int64_t f, unsigned char* dst, uint64_t* bar,
                                           uint64_t total_al, int rec_offset = 0) {
  const int64_t a0 = (int64_t)t * T;
  const int64_t a1 = min(L.ref.n_sel, a0 + T);
  const unsigned char* base = reinterpret_cast<const unsigned char*>(L.coords);
  const uint64_t b0 = (uint64_t)(f * L.n_atoms + a0) * STRIDE * 4ull;
  const uint64_t b1 = (uint64_t)(f * L.n_atoms + a1) * STRIDE * 4ull;
  const uint64_t c0 = b0 & ~15ull;
  uint64_t c1 = (b1 + 15ull) & ~15ull;
  if (c1 > total_al) {
    const uint64_t tail0 = total_al > c0 ? total_al : c0;
    for (uint64_t bb = tail0; bb < b1; bb += 4)
      *reinterpret_cast<float*>(dst + (bb - c0)) = __ldg(reinterpret_cast<const float*>(base + bb));
    c1 = tail0;
  }
  const uint32_t core = (uint32_t)(c1 - c0);
  // order this CTA's earlier generic-proxy reads of the stage before the
  // async-proxy write into it
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_arrive_expect_tx(bar, core + (rec_offset ? (uint32_t)(kStatDoubles * 8) : 0u));
  if (core) bulk_copy_g2s(dst, base + c0, core, bar);
  if (rec_offset) bulk_copy_g2s(dst + rec_offset, L.rot + f * kStatDoubles, kStatDoubles * 8, bar);
}

// Streaming kernel.  Items (tile t, frame f) are enumerated tile-major; each
// CTA owns the contiguous run [w0, w1) and walks it with incremental (t, f).
// Thread 0 doubles as the producer: at the top of item i it refills the stage
// that item i-1 used (all consumers passed item i-1's named barrier, so its
// reads are done) with item i + kStages - 1.
template <int STRIDE, int APT, int MODE, bool GATHER>
__global__ void __launch_bounds__(kThreads, 3) rmsd_frames_kernel(const FrameLaunch L) {
  using G = Geo<STRIDE, APT>;
  constexpr int T = G::kTile;
  constexpr int S = G::kStages;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::kBarOffset);
  double* red = reinterpret_cast<double*>(smem + G::kRedOffset);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::kAbortOffset);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t n_sel = L.ref.n_sel;
  const int64_t F = L.n_frames;
  const int n_tiles = (int)((n_sel + T - 1) / T);
  const int64_t W = (int64_t)n_tiles * F;
  const int64_t w0 = W * blockIdx.x / gridDim.x, w1 = W * (blockIdx.x + 1) / gridDim.x;
  const int64_t n_items = w1 - w0;
  const uint64_t total_al = ((uint64_t)F * (uint64_t)L.n_atoms * STRIDE * 4ull) & ~15ull;

  if (tid == 0) {
    if (!GATHER)
      for (int st = 0; st < S; ++st) mbar_init(&full[st], 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();

  // producer cursor (thread 0 only).  Under the error-path test the first
  // stage of CTA 0 is never armed (WaitCfg::withhold).
  int tp = (int)(w0 / F);
  int64_t fp = w0 - (int64_t)tp * F;
  int64_t issued = 0;
  const bool withheld = L.wait.withhold && blockIdx.x == 0;
  if (!GATHER && tid == 0) {
    for (; issued < S - 1 && issued < n_items; ++issued) {
      if (!(withheld && issued == 0))
        issue_item<STRIDE, T>(L, tp, fp, smem + (issued % S) * G::kStageBytes, &full[issued % S], total_al,
                              MODE == kBwd ? G::kRecOffset : 0);
      if (++fp == F) { fp = 0; ++tp; }
    }
  }

  double yr[APT][3];
  float wr[MODE == kFwdW ? APT : 1];
  uint32_t gidx[GATHER ? APT : 1];
  int t = (int)(w0 / F);
  int64_t f = w0 - (int64_t)t * F;
  int cur_tile = -1;
  int s = 0;
  uint32_t phase = 0;
  for (int64_t i = 0; i < n_items; ++i) {
    if (!GATHER && tid == 0 && issued < n_items) {
      const int sp = (int)(issued % S);
      if (!(withheld && issued == 0))
        issue_item<STRIDE, T>(L, tp, fp, smem + sp * G::kStageBytes, &full[sp], total_al,
                              MODE == kBwd ? G::kRecOffset : 0);
      ++issued;
      if (++fp == F) { fp = 0; ++tp; }
    }
    const int64_t a0 = (int64_t)t * T;
    const int len = (int)(min(n_sel, a0 + T) - a0);
    if (t != cur_tile) {
      cur_tile = t;
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        const int k = tid + j * kConsumerThreads;
        if (k < len) {
          const double* y = L.ref.yc + (a0 + k) * 3;
          yr[j][0] = __ldg(y + 0); yr[j][1] = __ldg(y + 1); yr[j][2] = __ldg(y + 2);
          if (MODE == kFwdW) wr[MODE == kFwdW ? j : 0] = __ldg(L.ref.w + a0 + k);
          if (GATHER) {
            uint32_t idx = L.sel ? __ldg(L.sel + a0 + k) : (uint32_t)(a0 + k);
            if ((int64_t)idx >= L.n_atoms) {  // bad device-side selection: report, read atom 0
              atomicOr(L.status, kStatusBadIndex);
              idx = 0;
            }
            gidx[GATHER ? j : 0] = idx;
          }
        } else {
          yr[j][0] = yr[j][1] = yr[j][2] = 0.0;
          if (MODE == kFwdW) wr[MODE == kFwdW ? j : 0] = 0.f;
          if (GATHER) gidx[GATHER ? j : 0] = 0;
        }
      }
    }
    const float* xs = nullptr;
    bool ok = true;
    if (!GATHER) {
      ok = mbar_wait(&full[s], phase, L.status, kStatusTimeoutFull, abort_flag, L.wait.limit_ns);
      xs = reinterpret_cast<const float*>(smem + s * G::kStageBytes) +
           (int)(((uint64_t)(f * L.n_atoms + a0) * STRIDE) & 3ull);
    }
    const float* frame = L.coords + (size_t)f * L.n_atoms * STRIDE;

    // Gathered atoms are loaded up front (independent global loads in flight);
    // staged atoms are read from shared memory right where they are used.
    float xg[GATHER ? APT : 1][3];
    if (GATHER) {
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        const int k = tid + j * kConsumerThreads;
        if (k < len) {
          const float* p = frame + (size_t)gidx[GATHER ? j : 0] * STRIDE;
          xg[GATHER ? j : 0][0] = __ldg(p + 0);
          xg[GATHER ? j : 0][1] = __ldg(p + 1);
          xg[GATHER ? j : 0][2] = __ldg(p + 2);
        } else {
          xg[GATHER ? j : 0][0] = xg[GATHER ? j : 0][1] = xg[GATHER ? j : 0][2] = 0.f;
        }
      }
    }
    auto load_x = [&](int j, float& a, float& b, float& c) {
      const int k = tid + j * kConsumerThreads;
      if (GATHER) {
        a = xg[GATHER ? j : 0][0]; b = xg[GATHER ? j : 0][1]; c = xg[GATHER ? j : 0][2];
      } else if (ok && k < len) {
        if (STRIDE == 4) {
          const float4 q = reinterpret_cast<const float4*>(xs)[k];
          a = q.x; b = q.y; c = q.z;
        } else {
          a = xs[k * 3 + 0]; b = xs[k * 3 + 1]; c = xs[k * 3 + 2];
        }
      } else {
        a = b = c = 0.f;
      }
    };

    if (MODE == kBwd) {
      if (ok) {
        // the staged copy of the frame's rotation record, or (gathered) the record itself
        const double* rt = GATHER ? L.rot + f * kStatDoubles
                                  : reinterpret_cast<const double*>(smem + s * G::kStageBytes + G::kRecOffset);
        double R[9], c[3];
#pragma unroll
        for (int e = 0; e < 9; ++e) R[e] = rt[e];
        c[0] = rt[9]; c[1] = rt[10]; c[2] = rt[11];
        const double scale = rt[12];
        float* gframe = L.grad + (size_t)f * L.n_atoms * 3;
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          const int k = tid + j * kConsumerThreads;
          float x0, x1, x2;
          load_x(j, x0, x1, x2);
          if (k < len) {
            const double ty0 = R[0] * yr[j][0] + R[3] * yr[j][1] + R[6] * yr[j][2];
            const double ty1 = R[1] * yr[j][0] + R[4] * yr[j][1] + R[7] * yr[j][2];
            const double ty2 = R[2] * yr[j][0] + R[5] * yr[j][1] + R[8] * yr[j][2];
            const size_t atom = GATHER ? (size_t)gidx[GATHER ? j : 0] : (size_t)(a0 + k);
            float* g = gframe + atom * 3;
            g[0] = (float)(scale * (((double)x0 - c[0]) - ty0));
            g[1] = (float)(scale * (((double)x1 - c[1]) - ty1));
            g[2] = (float)(scale * (((double)x2 - c[2]) - ty2));
          }
        }
      }
      named_barrier_sync(1, kConsumerThreads);  // stage s free for the producer
    } else {
      double acc[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[e] = 0.0;
      if (MODE == kFwdRaw) {
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          float x0, x1, x2;
          load_x(j, x0, x1, x2);
          // y = y_c + mean, rebuilt in FP64; x - y in FP64
          const double d0 = (double)x0 - (yr[j][0] + L.ref.mean[0]);
          const double d1 = (double)x1 - (yr[j][1] + L.ref.mean[1]);
          const double d2 = (double)x2 - (yr[j][2] + L.ref.mean[2]);
          const bool in = ok && tid + j * kConsumerThreads < len;
          acc[0] = fma(d0, in ? d0 : 0.0, acc[0]);
          acc[1] = fma(d1, in ? d1 : 0.0, acc[1]);
          acc[2] = fma(d2, in ? d2 : 0.0, acc[2]);
        }
        acc[0] += acc[1] + acc[2];
        acc[1] = acc[2] = 0.0;
      } else if (MODE == kFwdW) {
        // weighted: sum w x, sum w x_a^2, sum x (w y_c)^T (the weight is folded
        // into the stored reference)
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          float f0, f1, f2;
          load_x(j, f0, f1, f2);
          const double x0 = f0, x1 = f1, x2 = f2, w = wr[MODE == kFwdW ? j : 0];
          const double u0 = w * x0, u1 = w * x1, u2 = w * x2;
          acc[0] += u0; acc[1] += u1; acc[2] += u2;
          acc[3] = fma(u0, x0, acc[3]); acc[4] = fma(u1, x1, acc[4]); acc[5] = fma(u2, x2, acc[5]);
          acc[6] = fma(x0, yr[j][0], acc[6]);  acc[7] = fma(x0, yr[j][1], acc[7]);  acc[8] = fma(x0, yr[j][2], acc[8]);
          acc[9] = fma(x1, yr[j][0], acc[9]);  acc[10] = fma(x1, yr[j][1], acc[10]); acc[11] = fma(x1, yr[j][2], acc[11]);
          acc[12] = fma(x2, yr[j][0], acc[12]); acc[13] = fma(x2, yr[j][1], acc[13]); acc[14] = fma(x2, yr[j][2], acc[14]);
        }
      } else {
#pragma unroll
        for (int j = 0; j < APT; ++j) {
          float f0, f1, f2;
          load_x(j, f0, f1, f2);
          const double x0 = f0, x1 = f1, x2 = f2;
          acc[0] += x0; acc[1] += x1; acc[2] += x2;
          acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
          acc[6] = fma(x0, yr[j][0], acc[6]);  acc[7] = fma(x0, yr[j][1], acc[7]);  acc[8] = fma(x0, yr[j][2], acc[8]);
          acc[9] = fma(x1, yr[j][0], acc[9]);  acc[10] = fma(x1, yr[j][1], acc[10]); acc[11] = fma(x1, yr[j][2], acc[11]);
          acc[12] = fma(x2, yr[j][0], acc[12]); acc[13] = fma(x2, yr[j][1], acc[13]); acc[14] = fma(x2, yr[j][2], acc[14]);
        }
      }
      const double v = warp_reduce_scatter16(acc);
      double* rb = red + (i & 1) * (kConsumerWarps * 16);
      if ((lane & 1) == 0) rb[warp * 16 + (lane >> 1)] = v;
      named_barrier_sync(1, kConsumerThreads);  // also frees stage s for the producer
      if (warp == (int)(i & (kConsumerWarps - 1))) item_epilogue(L, rb, n_tiles, t, f);
    }
    if (*abort_flag) break;
    if (++s == S) { s = 0; phase ^= 1u; }
    if (++f == F) { f = 0; ++t; }
  }

  // every copy this CTA issued must land before the CTA may exit (a withheld
  // stage has none)
  if (!GATHER && tid == 0) {
    const int64_t first = issued > S ? issued - S : 0;
    for (int64_t j = first; j < issued; ++j)
      if (!(withheld && j == 0)) mbar_drain(&full[j % S], (uint32_t)((j / S) & 1), L.status);
  }
}

// Backward prologue: per frame, the rotation from the QCP eigenvector of the
// stored H, the centroid and the scale dL/drmsd / (n rmsd).
__global__ void rmsd_bwd_prologue(const double* __restrict__ stats, const float* __restrict__ grad_rmsd,
                                  const double* __restrict__ grad_f64, int64_t grad_stride, int64_t n_frames,
                                  double* __restrict__ rot) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_frames) return;
  const double* st = stats + f * kStatDoubles;
  double h[9], r[9];
  for (int e = 0; e < 9; ++e) h[e] = st[3 + e];
  rotation_from_qcp(h, st[12], r);
  const double rmsd = st[13], n = st[14];
  const double g = grad_f64 ? grad_f64[f * grad_stride] : grad_rmsd ? (double)grad_rmsd[f] : 1.0;
  const double scale = (rmsd > 0.0 && n > 0.0) ? g / (n * rmsd) : 0.0;
  double* o = rot + f * kStatDoubles;
  for (int e = 0; e < 9; ++e) o[e] = r[e];
  o[9] = st[0]; o[10] = st[1]; o[11] = st[2];
  o[12] = scale; o[13] = 0; o[14] = 0; o[15] = 0;
}

// Residual pass for flagged frames (near-zero RMSD): the RMSD from explicit
// residuals sum |R (x_k - x_bar) - (y_k - y_bar)|^2 in FP64, as the reference's
// rmsd_aligned_selected computes every frame (plan.rs:1223-1247), with R from
// the QCP eigenvector.  One CTA per flagged frame (grid-stride).
template <int STRIDE>
__global__ void __launch_bounds__(256) rmsd_refine_kernel(const FrameLaunch L) {
  __shared__ double sh_r[12];
  __shared__ double red[8];
  const unsigned count = *L.refine_count;
  const int64_t n_sel = L.ref.n_sel;
  const double inv_n = 1.0 / (double)n_sel;
  for (unsigned rix = blockIdx.x; rix < count; rix += gridDim.x) {
    const double* rec = L.refine + (size_t)rix * kStatDoubles;
    if (threadIdx.x == 0) {
      double h[9], r[9];
      for (int e = 0; e < 9; ++e) h[e] = rec[4 + e];
      rotation_from_qcp(h, rec[13], r);
      for (int e = 0; e < 9; ++e) sh_r[e] = r[e];
      sh_r[9] = rec[1]; sh_r[10] = rec[2]; sh_r[11] = rec[3];
    }
    __syncthreads();
    const int64_t f = (int64_t)rec[0];
    double R[9], c[3];
    for (int e = 0; e < 9; ++e) R[e] = sh_r[e];
    c[0] = sh_r[9]; c[1] = sh_r[10]; c[2] = sh_r[11];
    const double my0 = L.ref.sum_c[0] * inv_n, my1 = L.ref.sum_c[1] * inv_n, my2 = L.ref.sum_c[2] * inv_n;
    const float* frame = L.coords + (size_t)f * L.n_atoms * STRIDE;
    double acc = 0.0;
    for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
      int64_t atom = L.sel ? (int64_t)L.sel[k] : k;
      if (atom >= L.n_atoms) atom = 0;  // reported by the forward kernel
      const float* p = frame + atom * STRIDE;
      const double d0 = (double)p[0] - c[0], d1 = (double)p[1] - c[1], d2 = (double)p[2] - c[2];
      const double* y = L.ref.yc + k * 3;
      const double r0 = R[0] * d0 + R[1] * d1 + R[2] * d2 - (y[0] - my0);
      const double r1 = R[3] * d0 + R[4] * d1 + R[5] * d2 - (y[1] - my1);
      const double r2 = R[6] * d0 + R[7] * d1 + R[8] * d2 - (y[2] - my2);
      acc += r0 * r0 + r1 * r1 + r2 * r2;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += red[w];
      const double rmsd = sqrt(t * inv_n);
      if (L.out.rmsd) L.out.rmsd[f] = rmsd;
      if (L.out.stats) L.out.stats[f * kStatDoubles + 13] = rmsd;
    }
    __syncthreads();
  }
}

// Gathered forward statistics (a selection's scattered atoms, or frames whose
// base is not 16-byte aligned).  One warp per (tile, frame) item, tiles of
// kConsumerThreads * kApt list positions as in the streaming kernel, so the
// partial records and rmsd_finalize_kernel are shared.  No block barrier: a
// warp walks its contiguous run of items (tile-major, so a tile's indices and
// reference stay in L1 across frames) in sub-chunks of 32 x kGatherJ
// positions, all of a sub-chunk's loads in flight before any use, and
// reduces its sums with shuffles.  Latency is hidden by the warps resident
// per SM instead of by a CTA-wide pipeline.
//
// An atom's 12 bytes cost two loads, not three: an 8-byte load of the pair
// that starts on an 8-byte boundary (x,y or y,z) and a 4-byte load of the
// other coordinate.
constexpr int kGatherJ = 4;
constexpr int kGatherThreads = 128;

__device__ __forceinline__ void load_xyz(const float* p, float& x, float& y, float& z) {
  const bool odd = (reinterpret_cast<uintptr_t>(p) & 7u) != 0;
  const float2 pr = __ldg(reinterpret_cast<const float2*>(p + (odd ? 1 : 0)));
  const float s = __ldg(p + (odd ? 0 : 2));
  x = odd ? s : pr.x;
  y = odd ? pr.x : pr.y;
  z = odd ? pr.y : s;
}

template <int STRIDE, int MODE>
__global__ void __launch_bounds__(kGatherThreads) rmsd_gather_kernel(const FrameLaunch L, int tile) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * kGatherThreads + threadIdx.x) >> 5;
  const int64_t n_warps = (int64_t)gridDim.x * (kGatherThreads / 32);
  const int64_t n_sel = L.ref.n_sel;
  const int64_t F = L.n_frames;
  const int n_tiles = (int)((n_sel + tile - 1) / tile);
  const int64_t W = (int64_t)n_tiles * F;
  const int64_t w0 = W * gw / n_warps, w1 = W * (gw + 1) / n_warps;
  int t = (int)(w0 / F);
  int64_t f = w0 - (int64_t)t * F;
  for (int64_t w = w0; w < w1; ++w) {
    const int64_t a0 = (int64_t)t * tile;
    const int64_t a1 = min(n_sel, a0 + tile);
    const float* frame = L.coords + (size_t)f * L.n_atoms * STRIDE;
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
#pragma unroll 1
    for (int64_t c0 = a0; c0 < a1; c0 += 32 * kGatherJ) {
      float x[kGatherJ][3];
      double y[kGatherJ][3];
      float wt[MODE == kFwdW ? kGatherJ : 1];
#pragma unroll
      for (int j = 0; j < kGatherJ; ++j) {
        const int64_t k = c0 + lane + 32 * j;
        if (k < a1) {
          int64_t idx = L.sel ? (int64_t)__ldg(L.sel + k) : k;
          if (idx >= L.n_atoms) {  // bad device-side selection: report, read atom 0
            atomicOr(L.status, kStatusBadIndex);
            idx = 0;
          }
          load_xyz(frame + idx * STRIDE, x[j][0], x[j][1], x[j][2]);
          const double* yp = L.ref.yc + k * 3;
          y[j][0] = __ldg(yp); y[j][1] = __ldg(yp + 1); y[j][2] = __ldg(yp + 2);
          if (MODE == kFwdW) wt[MODE == kFwdW ? j : 0] = __ldg(L.ref.w + k);
        } else {
          x[j][0] = x[j][1] = x[j][2] = 0.f;
          y[j][0] = y[j][1] = y[j][2] = 0.0;
          if (MODE == kFwdW) wt[MODE == kFwdW ? j : 0] = 0.f;
        }
      }
#pragma unroll
      for (int j = 0; j < kGatherJ; ++j) {
        const double x0 = x[j][0], x1 = x[j][1], x2 = x[j][2];
        if (MODE == kFwdRaw) {
          if (c0 + lane + 32 * j < a1) {
            const double d0 = x0 - (y[j][0] + L.ref.mean[0]);
            const double d1 = x1 - (y[j][1] + L.ref.mean[1]);
            const double d2 = x2 - (y[j][2] + L.ref.mean[2]);
            acc[0] = fma(d0, d0, acc[0]);
            acc[1] = fma(d1, d1, acc[1]);
            acc[2] = fma(d2, d2, acc[2]);
          }
        } else {
          if (MODE == kFwdW) {
            const double wj = wt[MODE == kFwdW ? j : 0];
            const double u0 = wj * x0, u1 = wj * x1, u2 = wj * x2;
            acc[0] += u0; acc[1] += u1; acc[2] += u2;
            acc[3] = fma(u0, x0, acc[3]); acc[4] = fma(u1, x1, acc[4]); acc[5] = fma(u2, x2, acc[5]);
          } else {
            acc[0] += x0; acc[1] += x1; acc[2] += x2;
            acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
          }
          acc[6] = fma(x0, y[j][0], acc[6]);  acc[7] = fma(x0, y[j][1], acc[7]);  acc[8] = fma(x0, y[j][2], acc[8]);
          acc[9] = fma(x1, y[j][0], acc[9]);  acc[10] = fma(x1, y[j][1], acc[10]); acc[11] = fma(x1, y[j][2], acc[11]);
          acc[12] = fma(x2, y[j][0], acc[12]); acc[13] = fma(x2, y[j][1], acc[13]); acc[14] = fma(x2, y[j][2], acc[14]);
        }
      }
    }
    if (MODE == kFwdRaw) {
      acc[0] += acc[1] + acc[2];
      acc[1] = acc[2] = 0.0;
    }
    const double v = warp_reduce_scatter16(acc);
    if ((lane & 1) == 0) L.partial[((size_t)f * n_tiles + t) * kStatDoubles + (lane >> 1)] = v;
    if (++f == F) { f = 0; ++t; }
  }
}

// ---------------------------------------------------------------------------
// host-side launch helpers
// ---------------------------------------------------------------------------

template <int STRIDE, int MODE>
static cudaError_t launch_gather(const FrameLaunch& L, cudaStream_t s) {
  rmsd_gather_kernel<STRIDE, MODE><<<L.grid, kGatherThreads, 0, s>>>(L, L.tile_atoms);
  return cudaGetLastError();
}

template <int STRIDE>
static int gather_occupancy() {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, rmsd_gather_kernel<STRIDE, kFwdW>, kGatherThreads, 0) !=
      cudaSuccess)
    blocks = 4;
  return blocks < 1 ? 1 : blocks;
}

template <int STRIDE, int APT, int MODE, bool GATHER>
static cudaError_t launch_one(const FrameLaunch& L, cudaStream_t s) {
  using G = Geo<STRIDE, APT>;
  auto kern = rmsd_frames_kernel<STRIDE, APT, MODE, GATHER>;
  const size_t smem = GATHER ? (size_t)(G::kAbortOffset + 16) : (size_t)G::kSmemBytes;
  static bool attr_done[64] = {};  // per instantiation and device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  kern<<<L.grid, kThreads, smem, s>>>(L);
  return cudaGetLastError();
}

template <int STRIDE, int APT, int MODE, bool GATHER>
static int occupancy_one() {
  using G = Geo<STRIDE, APT>;
  auto kern = rmsd_frames_kernel<STRIDE, APT, MODE, GATHER>;
  const size_t smem = GATHER ? (size_t)(G::kAbortOffset + 16) : (size_t)G::kSmemBytes;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::kSmemBytes);
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kThreads, smem) != cudaSuccess) blocks = 1;
  return blocks < 1 ? 1 : blocks;
}

// Tile shape: 8 atoms per thread x 128 threads = 1024-atom tiles; the
// reference atoms of a tile live in registers (48 per thread).
constexpr int kApt = 8;

template <int MODE>
static cudaError_t dispatch(const FrameLaunch& L, cudaStream_t s) {
  if constexpr (MODE != kBwd) {
    if (L.gather) return L.stride == 4 ? launch_gather<4, MODE>(L, s) : launch_gather<3, MODE>(L, s);
  }
  if (L.stride == 4) return L.gather ? launch_one<4, kApt, MODE, true>(L, s) : launch_one<4, kApt, MODE, false>(L, s);
  return L.gather ? launch_one<3, kApt, MODE, true>(L, s) : launch_one<3, kApt, MODE, false>(L, s);
}

template <int MODE>
static int occupancy(const FrameLaunch& L) {
  if (L.stride == 4) return L.gather ? occupancy_one<4, kApt, MODE, true>() : occupancy_one<4, kApt, MODE, false>();
  return L.gather ? occupancy_one<3, kApt, MODE, true>() : occupancy_one<3, kApt, MODE, false>();
}

int frame_tiles(const FrameLaunch& L) {
  const int64_t n = L.lanes ? L.lane_atoms : L.ref.n_sel;
  return (int)((n + L.tile_atoms - 1) / L.tile_atoms);
}

size_t frame_smem_bytes(int stride, int tile_atoms) {
  (void)tile_atoms;
  return stride == 4 ? Geo<4, kApt>::kSmemBytes : Geo<3, kApt>::kSmemBytes;
}

void frame_plan(FrameLaunch& L, int sm_count) {
  // a dense selection streams itself; a gathered one only through an
  // expansion the caller prepared (lane_y set)
  if (!L.lane_y && !L.gather) {
    L.lane_atom0 = 0;
    L.lane_atoms = L.ref.n_sel;
    L.lane_y = L.ref.yc;
    L.lane_w = L.ref.w;
  }
  L.lanes = L.lane_y && lanes_eligible(L) && lanes_worthwhile(L, sm_count);
  L.tile_atoms = L.lanes ? lanes_tile(L, sm_count) : kConsumerThreads * kApt;
}

int frame_grid(const FrameLaunch& L, int sm_count, bool backward) {
  if (L.lanes && !backward) return lanes_grid(L, sm_count);
  if (L.gather && !backward) {
    static int gocc[2] = {};
    int& occ = gocc[L.stride == 4];
    if (occ == 0) occ = L.stride == 4 ? gather_occupancy<4>() : gather_occupancy<3>();
    const int64_t warps = (int64_t)frame_tiles(L) * L.n_frames;  // one warp per item at most
    const int64_t cap = (int64_t)sm_count * occ;
    return (int)std::max<int64_t>(1, std::min<int64_t>((warps + kGatherThreads / 32 - 1) / (kGatherThreads / 32), cap));
  }
  static int cache[2][2][2] = {};  // [bwd][stride4][gather]
  int& occ = cache[backward ? 1 : 0][L.stride == 4][L.gather ? 1 : 0];
  if (occ == 0) occ = backward ? occupancy<kBwd>(L) : occupancy<kFwdFit>(L);
  const int64_t items = (int64_t)frame_tiles(L) * L.n_frames;
  const int64_t cap = (int64_t)sm_count * occ;
  return (int)std::max<int64_t>(1, std::min<int64_t>(items, cap));
}

cudaError_t launch_rmsd_forward(const FrameLaunch& L, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  if (!L.align) {
    cudaError_t e = L.lanes ? launch_lanes_forward(L, true, s) : dispatch<kFwdRaw>(L, s);
    if (e != cudaSuccess) return e;
    rmsd_finalize_kernel<kFwdRaw><<<(unsigned)((L.n_frames + 7) / 8), 256, 0, s>>>(L, frame_tiles(L));
    return cudaGetLastError();
  }
  if (L.refine) {
    cudaError_t e = cudaMemsetAsync(L.refine_count, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = L.lanes ? launch_lanes_forward(L, false, s) : dispatch<kFwdFit>(L, s);
  if (e != cudaSuccess) return e;
  rmsd_finalize_kernel<kFwdFit><<<(unsigned)((L.n_frames + 7) / 8), 256, 0, s>>>(L, frame_tiles(L));
  if ((e = cudaGetLastError()) != cudaSuccess || !L.refine) return e;
  const int blocks = (int)std::min<int64_t>(L.n_frames, 148);
  if (L.stride == 4) rmsd_refine_kernel<4><<<blocks, 256, 0, s>>>(L);
  else rmsd_refine_kernel<3><<<blocks, 256, 0, s>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_gather_partials(const FrameLaunch& L, bool raw, int sm_count, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  FrameLaunch B = L;
  B.lanes = false;
  B.gather = true;
  B.grid = frame_grid(B, sm_count, false);
  const int mode = raw ? kFwdRaw : (L.ref.w ? kFwdW : kFwdFit);
  if (L.stride == 4) {
    if (mode == kFwdRaw) return launch_gather<4, kFwdRaw>(B, s);
    return mode == kFwdW ? launch_gather<4, kFwdW>(B, s) : launch_gather<4, kFwdFit>(B, s);
  }
  if (mode == kFwdRaw) return launch_gather<3, kFwdRaw>(B, s);
  return mode == kFwdW ? launch_gather<3, kFwdW>(B, s) : launch_gather<3, kFwdFit>(B, s);
}

cudaError_t launch_rmsd_stream(const FrameLaunch& L, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  return L.lanes ? launch_lanes_forward(L, false, s) : dispatch<kFwdFit>(L, s);
}

cudaError_t launch_rmsd_stream_weighted(const FrameLaunch& L, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  return L.lanes ? launch_lanes_forward(L, false, s) : dispatch<kFwdW>(L, s);
}

cudaError_t launch_rmsd_backward(const FrameLaunch& L, const double* stats, const float* grad_rmsd,
                                 const double* grad_f64, int64_t grad_stride, double* rot_scratch, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  const int threads = 128;
  const int blocks = (int)((L.n_frames + threads - 1) / threads);
  rmsd_bwd_prologue<<<blocks, threads, 0, s>>>(stats, grad_rmsd, grad_f64, grad_stride, L.n_frames, rot_scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  FrameLaunch B = L;
  B.rot = rot_scratch;
  return dispatch<kBwd>(B, s);
}

}  // namespace wmd

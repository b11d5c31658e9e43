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
//     (16 shuffles) and a 2 KB shared buffer.  Frames spanning several tiles
//     leave a 16-double partial in scratch; the CTA that completes a frame
//     (atomic counter) adds the partials in tile order -- so results are
//     bitwise reproducible -- runs QCP in FP64 and resets the counter.
//   * Bounded waits everywhere: a wait that exceeds kWaitLimitNs records a
//     status bit in the context's status word and the CTA exits after letting
//     its copies in flight land.
//
// The backward kernel streams the same items again, re-derives R from the QCP
// eigenvector of the stored H (a per-frame prologue kernel), and writes
// grad = dL/drmsd * (x - x_bar - R^T y_c) / (n rmsd) as float32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_util.cuh"
#include "qcp.cuh"
#include "wmd_internal.h"

namespace wmd {

enum Mode : int { kFwdFit = 0, kFwdRaw = 1, kBwd = 2 };

template <int STRIDE, int APT>
struct Geo {
  static constexpr int kTile = kConsumerThreads * APT;
  static constexpr int kStageBytes = ((kTile * STRIDE * 4 + 32) + 127) / 128 * 128;
  static constexpr int kStagesRaw = 98304 / kStageBytes;
  static constexpr int kStages = kStagesRaw < 2 ? 2 : (kStagesRaw > 8 ? 8 : kStagesRaw);
  static constexpr int kRedBytes = 2 * kConsumerWarps * 16 * 8;
  static constexpr int kBarOffset = kStages * kStageBytes;
  static constexpr int kRedOffset = kBarOffset + 2 * kStages * 8;
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

// Leader warp of an item: total over the 8 consumer warps, then either finish
// the frame or deposit a tile partial and let the last tile finish it.
__device__ __forceinline__ void item_epilogue(const FrameLaunch& L, const double* red, int n_tiles, int t,
                                              int64_t f, int mode) {
  const int lane = threadIdx.x & 31;
  double v = 0.0;
  if (lane < 16) {
#pragma unroll
    for (int w = 0; w < kConsumerWarps; ++w) v += red[w * 16 + lane];
  }
  if (n_tiles == 1) {
    finish_frame(L, f, v, mode);
    return;
  }
  double* part = L.partial + (size_t)f * n_tiles * kStatDoubles;
  if (lane < 16) part[(size_t)t * kStatDoubles + lane] = v;
  __threadfence();
  __syncwarp();
  unsigned prev = 0;
  if (lane == 0) prev = atomicAdd(L.counter + f, 1u);
  prev = __shfl_sync(0xffffffffu, prev, 0);
  if (prev != (unsigned)(n_tiles - 1)) return;
  __threadfence();
  double s = 0.0;
  if (lane < 16)
    for (int tt = 0; tt < n_tiles; ++tt) s += __ldcg(part + (size_t)tt * kStatDoubles + lane);
  if (lane == 0) L.counter[f] = 0u;
  finish_frame(L, f, s, mode);
}

template <int STRIDE, int APT, int MODE, bool GATHER>
__global__ void __maxnreg__(112) rmsd_frames_kernel(const FrameLaunch L) {
  using G = Geo<STRIDE, APT>;
  constexpr int T = G::kTile;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::kBarOffset);
  uint64_t* empty = full + G::kStages;
  double* red = reinterpret_cast<double*>(smem + G::kRedOffset);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::kAbortOffset);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n_sel = L.ref.n_sel;
  const int n_tiles = (int)((n_sel + T - 1) / T);
  const int64_t W = (int64_t)n_tiles * L.n_frames;
  const int64_t w0 = W * blockIdx.x / gridDim.x, w1 = W * (blockIdx.x + 1) / gridDim.x;

  if (!GATHER) {
    if (threadIdx.x == 0) {
      for (int s = 0; s < G::kStages; ++s) {
        mbar_init(&full[s], 1);
        mbar_init(&empty[s], kConsumerWarps);
      }
      *abort_flag = 0;
      fence_barrier_init();
    }
  } else if (threadIdx.x == 0) {
    *abort_flag = 0;
  }
  __syncthreads();

  if (warp == kConsumerWarps) {
    // ---------------- producer warp ----------------
    if (GATHER || lane != 0) return;
    const uint64_t total = (uint64_t)L.n_frames * (uint64_t)L.n_atoms * STRIDE * 4ull;
    const uint64_t total_al = total & ~15ull;
    const unsigned char* base = reinterpret_cast<const unsigned char*>(L.coords);
    int64_t i = 0;
    for (int64_t w = w0; w < w1; ++w, ++i) {
      const int s = (int)(i % G::kStages);
      const uint32_t ph = (uint32_t)((i / G::kStages) & 1);
      if (!mbar_wait(&empty[s], ph ^ 1u, L.status, kStatusTimeoutEmpty, abort_flag)) break;
      const int t = (int)(w / L.n_frames);
      const int64_t f = w - (int64_t)t * L.n_frames;
      const int64_t a0 = (int64_t)t * T;
      const int64_t a1 = min(n_sel, a0 + T);
      const uint64_t b0 = (uint64_t)(f * L.n_atoms + a0) * STRIDE * 4ull;
      const uint64_t b1 = (uint64_t)(f * L.n_atoms + a1) * STRIDE * 4ull;
      const uint64_t c0 = b0 & ~15ull;
      uint64_t c1 = (b1 + 15ull) & ~15ull;
      unsigned char* dst = smem + s * G::kStageBytes;
      if (c1 > total_al) {
        const uint64_t tail0 = total_al > c0 ? total_al : c0;
        for (uint64_t bb = tail0; bb < b1; bb += 4)
          *reinterpret_cast<float*>(dst + (bb - c0)) = __ldg(reinterpret_cast<const float*>(base + bb));
        c1 = tail0;
      }
      const uint32_t core = (uint32_t)(c1 - c0);
      mbar_arrive_expect_tx(&full[s], core);
      if (core) bulk_copy_g2s(dst, base + c0, core, &full[s]);
    }
    // let every copy this CTA issued land before the CTA may exit
    const int64_t n_issued = i;
    const int64_t first = n_issued > G::kStages ? n_issued - G::kStages : 0;
    for (int64_t j = first; j < n_issued; ++j) {
      const int s = (int)(j % G::kStages);
      const uint32_t ph = (uint32_t)((j / G::kStages) & 1);
      const uint64_t t0 = global_timer_ns();
      while (!mbar_try_wait(&full[s], ph)) {
        if (global_timer_ns() - t0 > kWaitLimitNs) {
          atomicOr(L.status, kStatusTimeoutDrain);
          break;
        }
      }
    }
    return;
  }

  // ---------------- consumer warps ----------------
  const int tid = threadIdx.x;  // 0 .. kConsumerThreads-1
  double yr[APT][3];
  uint32_t gidx[GATHER ? APT : 1];
  int cur_tile = -1;
  int64_t i = 0;
  for (int64_t w = w0; w < w1; ++w, ++i) {
    const int t = (int)(w / L.n_frames);
    const int64_t f = w - (int64_t)t * L.n_frames;
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
          if (GATHER) gidx[GATHER ? j : 0] = 0;
        }
      }
    }
    const float* xs = nullptr;
    int s = 0;
    bool ok = true;
    if (!GATHER) {
      s = (int)(i % G::kStages);
      const uint32_t ph = (uint32_t)((i / G::kStages) & 1);
      ok = mbar_wait(&full[s], ph, L.status, kStatusTimeoutFull, abort_flag);
      // The backward has no CTA barrier, so a failed wait can leave at once.  The
      // forward still joins this item's named barrier (with zero sums) and all
      // consumer warps then leave together on the shared abort flag.
      if (MODE == kBwd && !ok) break;
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
      const double* rt = L.rot + f * kStatDoubles;
      double R[9], c[3];
#pragma unroll
      for (int e = 0; e < 9; ++e) R[e] = __ldg(rt + e);
      c[0] = __ldg(rt + 9); c[1] = __ldg(rt + 10); c[2] = __ldg(rt + 11);
      const double scale = __ldg(rt + 12);
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
      if (!GATHER) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
      }
      continue;
    }

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
        const bool in = tid + j * kConsumerThreads < len;
        acc[0] = fma(d0, in ? d0 : 0.0, acc[0]);
        acc[1] = fma(d1, in ? d1 : 0.0, acc[1]);
        acc[2] = fma(d2, in ? d2 : 0.0, acc[2]);
      }
      acc[0] += acc[1] + acc[2];
      acc[1] = acc[2] = 0.0;
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
    if (!GATHER && ok) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    const double v = warp_reduce_scatter16(acc);
    double* rb = red + (i & 1) * (kConsumerWarps * 16);
    if ((lane & 1) == 0) rb[warp * 16 + (lane >> 1)] = v;
    named_barrier_sync(1, kConsumerThreads);
    if (*abort_flag) break;
    if (warp == (int)(i % kConsumerWarps)) item_epilogue(L, rb, n_tiles, t, f, MODE);
  }
}

// Backward prologue: per frame, the rotation from the QCP eigenvector of the
// stored H, the centroid and the scale dL/drmsd / (n rmsd).
__global__ void rmsd_bwd_prologue(const double* __restrict__ stats, const float* __restrict__ grad_rmsd,
                                  int64_t n_frames, double* __restrict__ rot) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_frames) return;
  const double* st = stats + f * kStatDoubles;
  double h[9], r[9];
  for (int e = 0; e < 9; ++e) h[e] = st[3 + e];
  rotation_from_qcp(h, st[12], r);
  const double rmsd = st[13], n = st[14];
  const double g = grad_rmsd ? (double)grad_rmsd[f] : 1.0;
  const double scale = (rmsd > 0.0 && n > 0.0) ? g / (n * rmsd) : 0.0;
  double* o = rot + f * kStatDoubles;
  for (int e = 0; e < 9; ++e) o[e] = r[e];
  o[9] = st[0]; o[10] = st[1]; o[11] = st[2];
  o[12] = scale; o[13] = 0; o[14] = 0; o[15] = 0;
}

// ---------------------------------------------------------------------------
// host-side launch helpers
// ---------------------------------------------------------------------------

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

// Tile shape: 4 atoms per consumer thread (1024-atom tiles) keeps the kernel
// within 112 registers, i.e. two CTAs (18 warps) per SM.
constexpr int kApt = 4;

template <int MODE>
static cudaError_t dispatch(const FrameLaunch& L, cudaStream_t s) {
  if (L.stride == 4) return L.gather ? launch_one<4, kApt, MODE, true>(L, s) : launch_one<4, kApt, MODE, false>(L, s);
  return L.gather ? launch_one<3, kApt, MODE, true>(L, s) : launch_one<3, kApt, MODE, false>(L, s);
}

template <int MODE>
static int occupancy(const FrameLaunch& L) {
  if (L.stride == 4) return L.gather ? occupancy_one<4, kApt, MODE, true>() : occupancy_one<4, kApt, MODE, false>();
  return L.gather ? occupancy_one<3, kApt, MODE, true>() : occupancy_one<3, kApt, MODE, false>();
}

int frame_tiles(const FrameLaunch& L) {
  return (int)((L.ref.n_sel + L.tile_atoms - 1) / L.tile_atoms);
}

size_t frame_smem_bytes(int stride, int tile_atoms) {
  (void)tile_atoms;
  return stride == 4 ? Geo<4, kApt>::kSmemBytes : Geo<3, kApt>::kSmemBytes;
}

int frame_grid(const FrameLaunch& L, int sm_count, bool backward) {
  static int cache[2][2][2] = {};  // [bwd][stride4][gather]
  int& occ = cache[backward ? 1 : 0][L.stride == 4][L.gather ? 1 : 0];
  if (occ == 0) occ = backward ? occupancy<kBwd>(L) : occupancy<kFwdFit>(L);
  const int64_t items = (int64_t)frame_tiles(L) * L.n_frames;
  const int64_t cap = (int64_t)sm_count * occ;
  return (int)std::max<int64_t>(1, std::min<int64_t>(items, cap));
}

cudaError_t launch_rmsd_forward(const FrameLaunch& L, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  return L.align ? dispatch<kFwdFit>(L, s) : dispatch<kFwdRaw>(L, s);
}

cudaError_t launch_rmsd_backward(const FrameLaunch& L, const double* stats, const float* grad_rmsd,
                                 double* rot_scratch, cudaStream_t s) {
  if (L.n_frames == 0) return cudaSuccess;
  const int threads = 128;
  const int blocks = (int)((L.n_frames + threads - 1) / threads);
  rmsd_bwd_prologue<<<blocks, threads, 0, s>>>(stats, grad_rmsd, L.n_frames, rot_scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  FrameLaunch B = L;
  B.rot = rot_scratch;
  return dispatch<kBwd>(B, s);
}

}  // namespace wmd

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
//   3. superpose_apply_staged (packed, aligned buffers) or
//      superpose_apply_kernel (the rest) moves every atom of every frame,
//      FP64 arithmetic rounded to float32 as the reference does.
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

// Staged apply for packed xyz input and output with 16-byte aligned bases:
// work items are (frame, 1024-atom chunk), frame-major; persistent CTAs walk
// contiguous runs.  Thread 0 streams each item's 16-byte hull into a 4-stage
// shared-memory ring (1-D bulk copies on mbarriers), every thread moves its
// atoms in place in the stage, and the item leaves by one bulk store of its
// aligned middle plus at most 2 x 3 scalar floats at its ends.  The stage of
// item i-1 is refilled at the end of item i, once its store has been read
// out (bulk wait_group.read).
constexpr int kApplyTile = 1024;
struct AGeo {
  static constexpr int kStageBytes = ((kApplyTile * 12 + 32) + 127) / 128 * 128;
  static constexpr int kStages = 4;
  static constexpr int kBarOffset = kStages * kStageBytes;
  static constexpr int kAbortOffset = kBarOffset + kStages * 8;
  static constexpr int kSmemBytes = kAbortOffset + 16;
};

__device__ __forceinline__ void apply_issue(const float* coords, int64_t n_frames, int64_t n_atoms, int64_t f, int c,
                                            unsigned char* dst, uint64_t* bar) {
  const int64_t a0 = (int64_t)c * kApplyTile;
  const int64_t a1 = min(n_atoms, a0 + kApplyTile);
  const unsigned char* base = reinterpret_cast<const unsigned char*>(coords);
  const uint64_t total_al = ((uint64_t)n_frames * (uint64_t)n_atoms * 12ull) & ~15ull;
  const uint64_t b0 = (uint64_t)(f * n_atoms + a0) * 12ull;
  const uint64_t b1 = (uint64_t)(f * n_atoms + a1) * 12ull;
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

__global__ void __launch_bounds__(kThreads, 4) superpose_apply_staged(const float* __restrict__ coords,
                                                                      int64_t n_frames, int64_t n_atoms,
                                                                      const double* __restrict__ xf,
                                                                      float* __restrict__ out, int* status) {
  constexpr int S = AGeo::kStages;
  constexpr int APT = kApplyTile / kConsumerThreads;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + AGeo::kBarOffset);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + AGeo::kAbortOffset);
  const int tid = threadIdx.x;
  const int nc = (int)((n_atoms + kApplyTile - 1) / kApplyTile);
  const int64_t W = (int64_t)nc * n_frames;
  const int64_t w0 = W * blockIdx.x / gridDim.x, w1 = W * (blockIdx.x + 1) / gridDim.x;
  const int64_t n_items = w1 - w0;
  if (tid == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&full[st], 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (n_items <= 0) return;
  int64_t pf = w0 / nc;
  int pc = (int)(w0 - pf * nc);
  int64_t issued = 0;
  auto issue = [&]() {
    const int sp = (int)(issued % S);
    apply_issue(coords, n_frames, n_atoms, pf, pc, smem + sp * AGeo::kStageBytes, &full[sp]);
    ++issued;
    if (++pc == nc) { pc = 0; ++pf; }
  };
  if (tid == 0)
    while (issued < S - 1 && issued < n_items) issue();
  int64_t f = w0 / nc;
  int c = (int)(w0 - f * nc);
  int64_t cur_f = -1;
  double R[9], t[3];
  int s = 0;
  uint32_t phase = 0;
  unsigned char* obase = reinterpret_cast<unsigned char*>(out);
  for (int64_t i = 0; i < n_items; ++i) {
    if (f != cur_f) {
      cur_f = f;
      const double* x = xf + f * kStatDoubles;
#pragma unroll
      for (int e = 0; e < 9; ++e) R[e] = __ldg(x + e);
      t[0] = __ldg(x + 9); t[1] = __ldg(x + 10); t[2] = __ldg(x + 11);
    }
    const int64_t a0 = (int64_t)c * kApplyTile;
    const int len = (int)(min(n_atoms, a0 + kApplyTile) - a0);
    const uint64_t b0 = (uint64_t)(f * n_atoms + a0) * 12ull;
    const bool ok = mbar_wait(&full[s], phase, status, kStatusTimeoutFull, abort_flag);
    float* xs = reinterpret_cast<float*>(smem + s * AGeo::kStageBytes) + (int)((b0 & 15ull) >> 2);
    if (ok) {
#pragma unroll
      for (int j = 0; j < APT; ++j) {
        const int k = tid + j * kConsumerThreads;
        if (k < len) {
          const double p0 = xs[k * 3 + 0], p1 = xs[k * 3 + 1], p2 = xs[k * 3 + 2];
          xs[k * 3 + 0] = (float)(R[0] * p0 + R[1] * p1 + R[2] * p2 + t[0]);
          xs[k * 3 + 1] = (float)(R[3] * p0 + R[4] * p1 + R[5] * p2 + t[1]);
          xs[k * 3 + 2] = (float)(R[6] * p0 + R[7] * p1 + R[8] * p2 + t[2]);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    named_barrier_sync(1, kConsumerThreads);
    const uint64_t b1 = b0 + (uint64_t)len * 12ull;
    const uint64_t m0 = (b0 + 15ull) & ~15ull, m1 = b1 & ~15ull;
    const bool mid = m1 > m0;
    const unsigned char* sbase = reinterpret_cast<const unsigned char*>(xs) - (b0 & 15ull);
    if (tid == 0) {
      if (ok && !*abort_flag && mid) bulk_copy_s2g(obase + m0, sbase + (m0 - (b0 & ~15ull)), (uint32_t)(m1 - m0));
      bulk_commit();
      bulk_wait_read<1>();
      if (issued < n_items) issue();
    } else if (ok && tid >= 32 && tid < 38) {
      const int q = tid - 32;
      const uint64_t at = mid ? (q < 3 ? b0 + 4ull * q : m1 + 4ull * (q - 3)) : b0 + 4ull * q;
      const uint64_t lim = mid ? (q < 3 ? m0 : b1) : b1;
      if (at < lim)
        *reinterpret_cast<float*>(obase + at) = *reinterpret_cast<const float*>(sbase + (at - (b0 & ~15ull)));
    }
    if (*abort_flag) break;
    if (++s == S) { s = 0; phase ^= 1u; }
    if (++c == nc) { c = 0; ++f; }
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
          atomicOr(status, kStatusTimeoutDrain);
          break;
        }
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
                                   const double* xf64, float* out, int sm_count, int* status, cudaStream_t s) {
  if (n_frames == 0 || n_atoms == 0) return cudaSuccess;
  const int64_t items = n_frames * ((n_atoms + 1023) / 1024);
  if (stride == 3 && ((reinterpret_cast<uintptr_t>(coords) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0) {
    static bool attr_done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_done[dev]) {
      cudaError_t e =
          cudaFuncSetAttribute(superpose_apply_staged, cudaFuncAttributeMaxDynamicSharedMemorySize, AGeo::kSmemBytes);
      if (e != cudaSuccess) return e;
      attr_done[dev] = true;
    }
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * 4));
    superpose_apply_staged<<<grid, kThreads, AGeo::kSmemBytes, s>>>(coords, n_frames, n_atoms, xf64, out, status);
    return cudaGetLastError();
  }
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * 8));
  if (stride == 4) superpose_apply_kernel<4><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, xf64, out);
  else superpose_apply_kernel<3><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, xf64, out);
  return cudaGetLastError();
}

}  // namespace wmd

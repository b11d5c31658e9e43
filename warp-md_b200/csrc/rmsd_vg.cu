// rmsd_vg.cu -- per-frame RMSD and dRMSD/dx in one kernel per frame group,
// for trajectories of many frames of up to kVgMaxAtoms atoms (packed xyz).
//
// The general path runs a statistics kernel (partials per (tile, frame) in
// global memory), a finalize kernel (QCP), a residual pass, a backward
// prologue (R from the eigenvector) and a gradient kernel: five launches and
// two round trips of per-frame records through memory.  Here one CTA owns a
// group of G <= 32 frames (lane l of every warp holds frame f0 + l, as in the
// frames-across-lanes kernel) and its 8 warps split the frames' atoms:
//
//   pass 1  each warp streams its atom slice of the G frames by 2-D TMA (three
//           [G rows x 128 B] boxes of packed xyz per 32-atom stage, 128-byte
//           swizzle, plus the 32 reference atoms by a 1-D bulk copy) through a
//           2-stage ring and adds, per lane and in FP64, the 15 sums of its
//           frame: sum x, sum x_a^2, sum x y_c^T;
//   combine the 8 warps' sums meet in shared memory (added in warp order, so
//           results are reproducible); warp 0 runs QCP in FP64, one frame per
//           lane, and the rotation R from the QCP eigenvector;
//   refine  frames with near-zero RMSD get the explicit FP64 residual sum
//           (a second pass over the group, only when such a frame exists);
//   pass 2  the warps stream their slices again (the group was read a few
//           microseconds earlier, so from L2 when it fits) and write
//           grad = w_f (x - x_bar - R^T y_c) / (n rmsd) in place in the
//           stage, which a 2-D TMA store sends to the gradient array.
//
// Three modes: forward (pass 1, QCP, refine: rmsd and the 16-double frame
// records of wmd_rmsd_forward), backward (pass 2 from those records: R is
// re-derived from the stored H and lambda) and both (value and gradient in one
// launch, x read from DRAM once: 12 B in + 12 B out per atom-frame).  The
// arithmetic is that of the general path (same sums, same QCP, same
// rotation), so the two agree to rounding.  No multicast loads anywhere.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "device_util.cuh"
#include "qcp.cuh"
#include "wmd_internal.h"

namespace wmd {

namespace {

constexpr int kVgWarps = 8;
constexpr int kVgThreads = kVgWarps * 32;
constexpr int kVgAtoms = 32;                          // atoms per stage
constexpr int kVgBoxBytes = 32 * 128;                 // smem per box: up to 32 rows of 128 bytes
constexpr int kVgXBytes = 3 * kVgBoxBytes;            // 32 atoms of packed xyz = 96 floats = 3 boxes
constexpr int kVgYBytes = kVgAtoms * 3 * 8;           // the stage's reference atoms, FP64
constexpr int kVgStageBytes = (kVgXBytes + kVgYBytes + 1023) / 1024 * 1024;
constexpr int kVgRingBytes = kVgWarps * 2 * kVgStageBytes;
constexpr double kVgKeepBytes = 100e6;              // frames held in L2 up to this size (126 MB L2)
constexpr int kDumpStride = 17;                       // doubles per lane in the combine (bank spread)
constexpr int kVgFrmOffset = kVgRingBytes;            // [32][16] doubles: per-frame R, x_bar, scale, flag
constexpr int kVgResOffset = kVgFrmOffset + 32 * 16 * 8;  // [8 warps][32] residual sums
constexpr int kVgBarOffset = kVgResOffset + kVgWarps * 32 * 8;
constexpr int kVgFlagOffset = kVgBarOffset + kVgWarps * 2 * 8;  // abort, any-refine, dump slot per warp
constexpr int kVgSmemBytes = kVgFlagOffset + 64 + 1024;  // + slack to align the base to 1024
static_assert(kDumpStride * 32 * 8 <= kVgStageBytes, "a warp's combine block fits one stage");

// frm record of one frame (doubles)
constexpr int kFrmR = 0, kFrmC = 9, kFrmScale = 12, kFrmFlag = 13;

struct VgArgs {
  int64_t F = 0, n_atoms = 0;
  int G = 32;                  // frames per group (TMA box rows)
  int64_t n_groups = 0;
  const double* yc = nullptr;  // [n_atoms + 32][3] centred reference, FP64, zero-padded
  double sum_c[3] = {0, 0, 0};
  double gy = 0;
  double* rmsd = nullptr;      // [F] or null
  double* stats = nullptr;     // [F][16]: written by forward, read by backward
  const void* w = nullptr;     // per-frame dL/drmsd, or null (1)
  int w_f64 = 0;               // w is double (else float)
  int64_t w_stride = 1;        // elements between frames' weights (0: one shared weight)
  int* status = nullptr;
  WaitCfg wait;
  int keep = 0;                // the frames fit L2: hold them for the next pass or kernel
};

// L2 eviction priorities (cache hints only): the frames a later pass of the
// group reads again are loaded evict_last, the last reads and the gradient
// stores evict_first, so that the gradient does not push the frames out of
// L2 between the passes.
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_normal() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar,
                                            uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// 2-D TMA store of a box from shared memory (bulk-group completion); elements
// outside the tensor are not written.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, const void* src, uint64_t policy) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group.L2::cache_hint [%0, {%1, %2}], [%3], %4;" ::
                   "l"(reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(smem_addr(src)), "l"(policy)
               : "memory");
}

__device__ __forceinline__ double frame_weight(const VgArgs& A, int64_t f) {
  if (!A.w) return 1.0;
  const int64_t i = f * A.w_stride;
  return A.w_f64 ? static_cast<const double*>(A.w)[i] : (double)static_cast<const float*>(A.w)[i];
}

// The 16-byte chunk c (0..23) of `lane`'s row in a stage: boxes of 32 floats
// (128 bytes) per row, 128-byte swizzle (chunk index XOR row mod 8).
__device__ __forceinline__ float4* stage_chunk(unsigned char* st, int lane, int c) {
  return reinterpret_cast<float4*>(st + (c >> 3) * kVgBoxBytes + lane * 128 + (((c & 7) ^ (lane & 7)) << 4));
}

template <int MODE>
__global__ void __launch_bounds__(kVgThreads, 1) rmsd_vg_kernel(const __grid_constant__ CUtensorMap mx,
                                                                const __grid_constant__ CUtensorMap mg,
                                                                const VgArgs A) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned char* ring = smem + warp * 2 * kVgStageBytes;
  double* frm = reinterpret_cast<double*>(smem + kVgFrmOffset);
  double* res = reinterpret_cast<double*>(smem + kVgResOffset);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kVgBarOffset);
  uint64_t* full = bars + warp * 2;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + kVgFlagOffset);
  volatile int* any_flag = abort_flag + 1;
  volatile int* dump_slot = abort_flag + 2;  // [kVgWarps]

  const int64_t S = (A.n_atoms + kVgAtoms - 1) / kVgAtoms;  // stages per frame
  const int64_t s0 = S * warp / kVgWarps, s1 = S * (warp + 1) / kVgWarps;
  const int64_t len = s1 - s0;
  const double n = (double)A.n_atoms, inv_n = 1.0 / n;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kVgWarps * 2; ++i) mbar_init(&bars[i], 1);
    *abort_flag = 0;
    *any_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();

  // Ring counters: loads issued (lane 0) and stages consumed (all lanes).
  // Under the error-path test warp 0 of CTA 0 never arms its first load.
  const bool withheld = A.wait.withhold && blockIdx.x == 0 && warp == 0;
  uint32_t n_iss = 0, n_don = 0;

  // pass 1 loads: held in L2 for pass 2 (both), or for the backward kernel
  // when the frames fit (forward); every other load is the last read
  const uint64_t pol_first = policy_evict_first();
  const uint64_t pol_hold = A.keep ? policy_evict_last() : policy_evict_normal();
  uint64_t pol_load = MODE == kVgBwd ? pol_first : pol_hold;

  auto issue = [&](int64_t s, int64_t f0) {  // lane 0: stage s of the group at frame f0
    const int slot = (int)(n_iss & 1u);
    unsigned char* dst = ring + slot * kVgStageBytes;
    if (!(withheld && n_iss == 0)) {
      // the gradient store that read this slot must be done reading it
      if (MODE != kVgFwd) bulk_wait_read<0>();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&full[slot], 3u * 128u * (uint32_t)A.G + (uint32_t)kVgYBytes);
#pragma unroll
      for (int b = 0; b < 3; ++b)
        tma_load_2d(dst + b * kVgBoxBytes, &mx, (int)(s * 96 + 32 * b), (int)f0, &full[slot], pol_load);
      bulk_copy_g2s(dst + kVgXBytes, A.yc + s * kVgAtoms * 3, kVgYBytes, &full[slot]);
    }
    ++n_iss;
  };

  // One pass of this warp over its stages; `pre` of them were issued already.
  // body(stage, stage index) runs on every lane.  Returns false when a wait
  // ran out (all lanes of the warp agree).  A slot is refilled as soon as the
  // warp is done with it, except in a pass that stores from its stages
  // (late): there stage k + 1 is loaded into the slot of stage k - 1 once
  // stage k has arrived, so that stage k - 1's store had that wait to finish
  // reading the slot.
  auto run_pass = [&](int64_t f0, int pre, bool late, auto&& body) -> bool {
    if (lane == 0)
      for (int64_t k = pre; k < (len < 2 ? len : (int64_t)2); ++k) issue(s0 + k, f0);
    for (int64_t k = 0; k < len; ++k) {
      bool ok = mbar_wait(&full[n_don & 1u], (n_don >> 1) & 1u, A.status, kStatusTimeoutFull, abort_flag,
                          A.wait.limit_ns);
      if (!__all_sync(0xffffffffu, ok)) return false;
      if (late && lane == 0 && k >= 1 && k + 1 < len) issue(s0 + k + 1, f0);
      body(ring + (n_don & 1u) * kVgStageBytes, s0 + k);
      ++n_don;
      __syncwarp();
      if (!late && lane == 0 && k + 2 < len) issue(s0 + k + 2, f0);
    }
    return true;
  };

  for (int64_t g = blockIdx.x; g < A.n_groups; g += gridDim.x) {
    const int64_t f0 = g * A.G;
    const int rows = (int)(A.F - f0 < (int64_t)A.G ? A.F - f0 : (int64_t)A.G);
    if (MODE != kVgBwd) pol_load = pol_hold;
    const bool mine = lane < rows;  // this lane's frame exists
    const int64_t f = f0 + lane;
    int pre = 0;  // stages of the next pass already issued

    // ---------------- pass 1: statistics (forward, both) ----------------
    if (MODE != kVgBwd) {
      double acc[15];
#pragma unroll
      for (int e = 0; e < 15; ++e) acc[e] = 0.0;
      const bool ok = run_pass(f0, 0, false, [&](unsigned char* st, int64_t) {
        const double2* yb = reinterpret_cast<const double2*>(st + kVgXBytes);
        auto add = [&](float fx, float fy, float fz, double y0, double y1, double y2) {
          const double x0 = fx, x1 = fy, x2 = fz;
          acc[0] += x0; acc[1] += x1; acc[2] += x2;
          acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
          acc[6] = fma(x0, y0, acc[6]);  acc[7] = fma(x0, y1, acc[7]);  acc[8] = fma(x0, y2, acc[8]);
          acc[9] = fma(x1, y0, acc[9]);  acc[10] = fma(x1, y1, acc[10]); acc[11] = fma(x1, y2, acc[11]);
          acc[12] = fma(x2, y0, acc[12]); acc[13] = fma(x2, y1, acc[13]); acc[14] = fma(x2, y2, acc[14]);
        };
        // atoms past the frame's end arrive as zeros against zero reference
        // rows, so they add nothing
        // the row's 24 chunks first: independent loads, then the arithmetic
        float4 v[24];
#pragma unroll
        for (int q = 0; q < 24; ++q) v[q] = *stage_chunk(st, lane, q);
#pragma unroll
        for (int m = 0; m < kVgAtoms / 4; ++m) {
          const float4 a = v[3 * m], b = v[3 * m + 1], c = v[3 * m + 2];
          const double2 y01 = yb[6 * m + 0], y23 = yb[6 * m + 1], y45 = yb[6 * m + 2];
          const double2 y67 = yb[6 * m + 3], y89 = yb[6 * m + 4], yab = yb[6 * m + 5];
          add(a.x, a.y, a.z, y01.x, y01.y, y23.x);
          add(a.w, b.x, b.y, y23.y, y45.x, y45.y);
          add(b.z, b.w, c.x, y67.x, y67.y, y89.x);
          add(c.y, c.z, c.w, y89.y, yab.x, yab.y);
        }
      });
      // both: prefetch the first stage of the next pass (every later pass of
      // the group streams the same stages in the same order), its last read
      pol_load = pol_first;
      if (MODE == kVgBoth && ok && len > 0) {
        if (lane == 0) issue(s0, f0);
        pre = 1;
      }
      // the warp's sums go to the slot its next load will use
      const int slot = (int)((n_don + (uint32_t)pre) & 1u);
      double* dump = reinterpret_cast<double*>(ring + slot * kVgStageBytes);
#pragma unroll
      for (int e = 0; e < 15; ++e) dump[lane * kDumpStride + e] = acc[e];
      if (lane == 0) dump_slot[warp] = slot;
    }
    __syncthreads();
    if (*abort_flag) break;

    // ---------------- per-frame records, one frame per lane of warp 0 ----------------
    if (warp == 0) {
      double R[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, c[3] = {0, 0, 0}, scale = 0.0;
      bool flag = false;
      if (MODE != kVgBwd) {
        double t[15];
#pragma unroll
        for (int e = 0; e < 15; ++e) t[e] = 0.0;
        for (int w = 0; w < kVgWarps; ++w) {  // warp order: reproducible sums
          const double* d =
              reinterpret_cast<const double*>(smem + (w * 2 + dump_slot[w]) * kVgStageBytes) + lane * kDumpStride;
#pragma unroll
          for (int e = 0; e < 15; ++e) t[e] += d[e];
        }
        if (mine) {
          const double sx[3] = {t[0], t[1], t[2]};
          double h[9];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) h[a * 3 + b] = t[6 + a * 3 + b] - sx[a] * A.sum_c[b] * inv_n;
          const double gx = t[3] + t[4] + t[5] - (sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]) * inv_n;
          const QcpOut q = qcp_lambda(h, 0.5 * (gx + A.gy));
          const double rmsd = sqrt(msd_from(gx, A.gy, q.lambda, n));
          flag = rmsd < kRefineScale * (gx + A.gy) * inv_n;
          if (A.rmsd) A.rmsd[f] = rmsd;
          if (A.stats) {
            double* st = A.stats + f * kStatDoubles;
            st[0] = sx[0] * inv_n; st[1] = sx[1] * inv_n; st[2] = sx[2] * inv_n;
#pragma unroll
            for (int e = 0; e < 9; ++e) st[3 + e] = h[e];
            st[12] = q.lambda; st[13] = rmsd; st[14] = n; st[15] = gx + A.gy;
          }
          c[0] = sx[0] * inv_n; c[1] = sx[1] * inv_n; c[2] = sx[2] * inv_n;
          if (MODE == kVgBoth || flag) rotation_from_qcp(h, q.lambda, R);
          if (MODE == kVgBoth && !flag && rmsd > 0.0) scale = frame_weight(A, f) / (n * rmsd);
        }
      } else if (mine) {
        // backward: the forward's record (x_bar, H, lambda, rmsd, n)
        const double* st = A.stats + f * kStatDoubles;
        double h[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) h[e] = st[3 + e];
        rotation_from_qcp(h, st[12], R);
        c[0] = st[0]; c[1] = st[1]; c[2] = st[2];
        const double rmsd = st[13], nn = st[14];
        scale = (rmsd > 0.0 && nn > 0.0) ? frame_weight(A, f) / (nn * rmsd) : 0.0;
      }
      double* fr = frm + lane * 16;
#pragma unroll
      for (int e = 0; e < 9; ++e) fr[kFrmR + e] = R[e];
      fr[kFrmC + 0] = c[0]; fr[kFrmC + 1] = c[1]; fr[kFrmC + 2] = c[2];
      fr[kFrmScale] = scale;
      fr[kFrmFlag] = flag ? 1.0 : 0.0;
      const unsigned flags = __ballot_sync(0xffffffffu, flag);
      if (lane == 0) *any_flag = flags != 0u;
    }
    // the combine slots are loaded by TMA again after this barrier
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    // ---------------- explicit residuals for near-zero frames (rare) ----------------
    if (MODE != kVgBwd && *any_flag) {
      const double* fr = frm + lane * 16;
      double R[9], c[3];
#pragma unroll
      for (int e = 0; e < 9; ++e) R[e] = fr[kFrmR + e];
      c[0] = fr[kFrmC]; c[1] = fr[kFrmC + 1]; c[2] = fr[kFrmC + 2];
      const bool flag = fr[kFrmFlag] != 0.0;
      const double my0 = A.sum_c[0] * inv_n, my1 = A.sum_c[1] * inv_n, my2 = A.sum_c[2] * inv_n;
      double ra = 0.0;
      run_pass(f0, pre, false, [&](unsigned char* st, int64_t s) {
        const double2* yb = reinterpret_cast<const double2*>(st + kVgXBytes);
        const int valid = (int)(A.n_atoms - s * kVgAtoms < kVgAtoms ? A.n_atoms - s * kVgAtoms : (int64_t)kVgAtoms);
        auto add = [&](float fx, float fy, float fz, double y0, double y1, double y2, int k) {
          const double d0 = (double)fx - c[0], d1 = (double)fy - c[1], d2 = (double)fz - c[2];
          const double r0 = R[0] * d0 + R[1] * d1 + R[2] * d2 - (y0 - my0);
          const double r1 = R[3] * d0 + R[4] * d1 + R[5] * d2 - (y1 - my1);
          const double r2 = R[6] * d0 + R[7] * d1 + R[8] * d2 - (y2 - my2);
          if (flag && k < valid) ra += r0 * r0 + r1 * r1 + r2 * r2;
        };
#pragma unroll 1
        for (int m = 0; m < kVgAtoms / 4; ++m) {
          const float4 a = *stage_chunk(st, lane, 3 * m), b = *stage_chunk(st, lane, 3 * m + 1),
                       cc = *stage_chunk(st, lane, 3 * m + 2);
          const double2 y01 = yb[6 * m + 0], y23 = yb[6 * m + 1], y45 = yb[6 * m + 2];
          const double2 y67 = yb[6 * m + 3], y89 = yb[6 * m + 4], yab = yb[6 * m + 5];
          add(a.x, a.y, a.z, y01.x, y01.y, y23.x, 4 * m);
          add(a.w, b.x, b.y, y23.y, y45.x, y45.y, 4 * m + 1);
          add(b.z, b.w, cc.x, y67.x, y67.y, y89.x, 4 * m + 2);
          add(cc.y, cc.z, cc.w, y89.y, yab.x, yab.y, 4 * m + 3);
        }
      });
      pre = 0;  // the prefetched stage went to this pass
      res[warp * 32 + lane] = ra;
      __syncthreads();
      if (*abort_flag) break;
      if (warp == 0 && mine && flag) {
        double tot = 0.0;
        for (int w = 0; w < kVgWarps; ++w) tot += res[w * 32 + lane];
        const double rmsd = sqrt(tot * inv_n);
        if (A.rmsd) A.rmsd[f] = rmsd;
        if (A.stats) A.stats[f * kStatDoubles + 13] = rmsd;
        if (MODE == kVgBoth) frm[lane * 16 + kFrmScale] = rmsd > 0.0 ? frame_weight(A, f) / (n * rmsd) : 0.0;
      }
      __syncthreads();
    }

    // ---------------- pass 2: gradient (backward, both) ----------------
    if (MODE != kVgFwd) {
      const double* fr = frm + lane * 16;
      double R[9], c[3];
#pragma unroll
      for (int e = 0; e < 9; ++e) R[e] = fr[kFrmR + e];
      c[0] = fr[kFrmC]; c[1] = fr[kFrmC + 1]; c[2] = fr[kFrmC + 2];
      const double scale = fr[kFrmScale];
      // grad_a = scale x_a + t_a with t_a = -scale c_a - sum_b scale R_ba y_b:
      // 12 FP64 operations per atom (FP64 rounding differs from
      // scale (x - c - R^T y) by ~1e-14 relative, far below float32)
      double mt[9], d[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        d[a] = -scale * c[a];
#pragma unroll
        for (int b = 0; b < 3; ++b) mt[a * 3 + b] = -scale * R[b * 3 + a];
      }
      run_pass(f0, pre, true, [&](unsigned char* st, int64_t s) {
        const double2* yb = reinterpret_cast<const double2*>(st + kVgXBytes);
        auto grad3 = [&](float& fx, float& fy, float& fz, double y0, double y1, double y2) {
          const double t0 = fma(mt[2], y2, fma(mt[1], y1, fma(mt[0], y0, d[0])));
          const double t1 = fma(mt[5], y2, fma(mt[4], y1, fma(mt[3], y0, d[1])));
          const double t2 = fma(mt[8], y2, fma(mt[7], y1, fma(mt[6], y0, d[2])));
          fx = (float)fma(scale, (double)fx, t0);
          fy = (float)fma(scale, (double)fy, t1);
          fz = (float)fma(scale, (double)fz, t2);
        };
        // all loads of the row, then the arithmetic, then all stores back in
        // place: no load waits behind a store it might alias
        float4 v[24];
#pragma unroll
        for (int q = 0; q < 24; ++q) v[q] = *stage_chunk(st, lane, q);
#pragma unroll
        for (int m = 0; m < kVgAtoms / 4; ++m) {
          const double2 y01 = yb[6 * m + 0], y23 = yb[6 * m + 1], y45 = yb[6 * m + 2];
          const double2 y67 = yb[6 * m + 3], y89 = yb[6 * m + 4], yab = yb[6 * m + 5];
          float4& a = v[3 * m];
          float4& b = v[3 * m + 1];
          float4& cc = v[3 * m + 2];
          grad3(a.x, a.y, a.z, y01.x, y01.y, y23.x);
          grad3(a.w, b.x, b.y, y23.y, y45.x, y45.y);
          grad3(b.z, b.w, cc.x, y67.x, y67.y, y89.x);
          grad3(cc.y, cc.z, cc.w, y89.y, yab.x, yab.y);
        }
#pragma unroll
        for (int q = 0; q < 24; ++q) *stage_chunk(st, lane, q) = v[q];
        // the gradient of the stage leaves by TMA store (rows past the last
        // frame and atoms past the frame's end are outside the tensor)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
#pragma unroll
          for (int b = 0; b < 3; ++b)  // a box that starts past the frame's end has nothing to store
            if (s * 96 + 32 * b < A.n_atoms * 3)
              tma_store_2d(&mg, (int)(s * 96 + 32 * b), (int)f0, st + b * kVgBoxBytes, pol_first);
          bulk_commit();
        }
      });
      pre = 0;
    }
    __syncthreads();  // frm, res and the combine slots are rewritten by the next group
    if (*abort_flag) break;
  }

  if (lane == 0) {
    // after an abort, loads this warp issued may still be landing (a
    // withheld stage has none); stores must finish before the CTA exits
    for (uint32_t j = n_don; j < n_iss; ++j)
      if (!(withheld && j == 0)) mbar_drain(&full[j & 1u], (j >> 1) & 1u, A.status);
    if (MODE != kVgFwd) bulk_wait_all<0>();
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled vg_encode_fn() {
  static EncodeTiled fn = nullptr;
  if (fn) return fn;
  void* p = nullptr;
  cudaDriverEntryPointQueryResult qr;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) != cudaSuccess ||
      qr != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    return nullptr;
  }
  fn = reinterpret_cast<EncodeTiled>(p);
  return fn;
}

// [F rows][n_atoms * 3 floats] with a [G rows][32 floats] box, 128-byte swizzle.
// On failure *why describes the call.
bool encode_frames(CUtensorMap* map, const float* base, int64_t F, int64_t n_atoms, int G, const char* what,
                   const char** why) {
  static thread_local char msg[256];
  EncodeTiled enc = vg_encode_fn();
  if (!enc) {
    if (why) *why = "cuTensorMapEncodeTiled unavailable";
    return false;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)(n_atoms * 3), (cuuint64_t)F};
  const cuuint64_t strides[1] = {(cuuint64_t)(n_atoms * 12)};
  const cuuint32_t box[2] = {32, (cuuint32_t)G};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS && why) {
    snprintf(msg, sizeof(msg), "tensor map of the %s (CUresult %d, base %p, %lld x %lld floats, row %lld B, box 32 x %d)",
             what, (int)r, (const void*)base, (long long)(n_atoms * 3), (long long)F, (long long)(n_atoms * 12), G);
    *why = msg;
  }
  return r == CUDA_SUCCESS;
}

template <int MODE>
cudaError_t launch_mode(const CUtensorMap& mx, const CUtensorMap& mg, const VgArgs& A, int grid, cudaStream_t s) {
  auto kern = rmsd_vg_kernel<MODE>;
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kVgSmemBytes);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  kern<<<grid, kVgThreads, kVgSmemBytes, s>>>(mx, mg, A);
  return cudaGetLastError();
}

}  // namespace

bool vg_usable(const float* coords, const float* grad, int64_t n_frames, int64_t n_atoms, int stride, int sm_count) {
  static int mode = -1;
  if (mode < 0) {
    const char* e = std::getenv("WMD_VG");
    mode = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
  }
  if (!mode || stride != 3 || n_atoms < 4 || (n_atoms & 3) != 0 || n_atoms > kVgMaxAtoms) return false;
  // enough frames for full groups on every SM (whole-frame work per CTA)
  if (n_frames < 16 * (int64_t)sm_count || n_frames >= (int64_t(1) << 31)) return false;
  if ((reinterpret_cast<uintptr_t>(coords) & 15u) != 0) return false;
  if (grad && (reinterpret_cast<uintptr_t>(grad) & 15u) != 0) return false;
  return true;
}

cudaError_t launch_vg(int mode, const VgLaunch& V, int sm_count, cudaStream_t s, const char** why) {
  if (V.n_frames == 0) return cudaSuccess;
  // G frames per group: the fewest equal rounds of at most 32-frame groups
  // over one CTA per SM
  const int64_t sms = std::max(1, sm_count);
  const int64_t rounds = (V.n_frames + 32 * sms - 1) / (32 * sms);
  const int G = (int)std::min<int64_t>(32, (V.n_frames + sms * rounds - 1) / (sms * rounds));
  VgArgs A;
  A.F = V.n_frames;
  A.n_atoms = V.n_atoms;
  A.G = G;
  A.n_groups = (V.n_frames + G - 1) / G;
  A.yc = V.ref.yc;
  for (int c = 0; c < 3; ++c) A.sum_c[c] = V.ref.sum_c[c];
  A.gy = V.ref.gy;
  A.rmsd = V.rmsd;
  A.stats = V.stats;
  A.w = V.w;
  A.w_f64 = V.w_f64;
  A.w_stride = V.w_stride;
  A.status = V.status;
  A.wait = V.wait;
  // frames that fit comfortably in L2 are held there for the next pass (both)
  // or for the backward kernel that usually follows the forward
  A.keep = (double)V.n_frames * (double)V.n_atoms * 12.0 <= kVgKeepBytes;
  CUtensorMap mx, mg;
  if (!encode_frames(&mx, V.coords, V.n_frames, V.n_atoms, G, "frames", why)) return cudaErrorInvalidValue;
  if (mode != kVgFwd) {
    if (!encode_frames(&mg, V.grad, V.n_frames, V.n_atoms, G, "gradient", why)) return cudaErrorInvalidValue;
  } else {
    mg = mx;
  }
  if (why) *why = "kernel launch";
  const int grid = (int)std::min<int64_t>(A.n_groups, sms);
  if (mode == kVgFwd) return launch_mode<kVgFwd>(mx, mg, A, grid, s);
  if (mode == kVgBwd) return launch_mode<kVgBwd>(mx, mg, A, grid, s);
  return launch_mode<kVgBoth>(mx, mg, A, grid, s);
}

}  // namespace wmd

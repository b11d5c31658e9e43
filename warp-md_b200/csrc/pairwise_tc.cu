// pairwise_tc.cu -- all-pairs RMSD matrix on the tcgen05 tensor cores.
//
// Arithmetic.  Each frame is centred in FP64 and quantised to fixed point with
// one scale s for the whole trajectory: q = round((x - c) / s), |q| <= qmax
// (24-bit: qmax = 2^23 - 2^16; 16-bit: 2^15 - 2^8).  q is split into signed
// int8 limbs q = sum_p a_p 2^(8p) (balanced digits in [-128, 127]).  The
// covariance of a frame pair is then
//     H_ij = s^2 sum_{p,r} 2^(8(p+r)) sum_k a_p(i,k) a_r(j,k),
// i.e. "shift groups" g = p + r of int8 x int8 GEMMs whose int32 accumulation
// is exact (3 n 128^2 < 2^31 for n < 43,690 atoms), combined exactly in int64
// by the FP64 epilogue, which runs QCP per pair.  Split-BF16 with FP32
// accumulation cannot reach this: dropping or rounding the lo*lo products
// biases n*MSD by ~n |lo|^2, which at 1,000 atoms is ~1e-2 A in RMSD for
// adjacent frames.
//   2 limbs (16-bit): all four products, 3 groups -- the exact Gram matrix of
//       the quantised frames.
//   3 limbs (24-bit): the eight products other than lo x lo, 4 groups (1..4).
//       The frame self-sums G use the same truncated product, so a frame
//       against itself still gives exactly 0, and the truncation lowers n*MSD
//       by sum_k |lo_i - R lo_j|^2 s^2 (lo: the low limb, |lo| s < 7.7e-4 A at
//       100 A extent), about 1.2e-6 A^2 per atom: < 6e-5 A of RMSD above
//       0.01 A.  Pairs below 0.01 A are recomputed exactly in FP64 from the
//       coordinates (pair_refine_kernel), so every entry stays within 1e-4 A.
//
// Layout.  Rows of the GEMM are (frame, component); 10 frames occupy 32 rows
// (30 used), so a 128-row tile holds 40 frames and a frame's three rows sit in
// one warp's TMEM lane quarter.  The limb array is L[limb][row][k] (k = atom,
// padded to 64) and serves as both A (tile of 128 rows = 40 frames) and B
// (128 rows = 40 frames); D = A B^T, both operands K-major, M = N = 128 (an
// N of 128 or more runs the MMA at the full int8 rate with both operands in
// shared memory; N = 96 measured 86 % of it).
//
// Kernel.  Persistent, one CTA per SM, warp-specialised:
//   warp 0     TMA producer: per K chunk (32 atoms with 3 limbs, 64 with 2)
//              one 3-D box per operand (all limbs at once), SWIZZLE_32B or
//              SWIZZLE_64B, 4- or 3-stage mbarrier ring;
//   warp 1     allocates 512 TMEM columns; lane 0 issues tcgen05.mma
//              kind::i8 (M=128, N=128, K=32) for every limb pair into the
//              pair's shift-group accumulator (4 x 128 columns for 3 limbs,
//              3 x 128 for 2), commits stages back to the producer and tiles
//              to the epilogue;
//   warps 2-17 drain: tcgen05.ld of its 32 lanes x 32 columns per group,
//              exact combination of the groups in int64, the 9 entries of H
//              of its 10 x 10 frame pairs staged pair-major in shared memory,
//              release of TMEM (the next tile's MMAs start);
//   warps 18-21 stage the tile's per-frame terms (G, centroids);
//   warps 2-21 then run the FP64 pair epilogue (QCP) for the tile's 1,600
//              pairs, one pair per lane per round, and the symmetric store.
// Every wait is bounded; a wait that runs out raises the CTA's abort flag and
// all roles leave, after the MMAs in flight are drained and TMEM is freed.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/warpmd_rmsd.h"
#include "device_util.cuh"
#include "pairwise_tc.h"
#include "qcp.cuh"

namespace wmd {
namespace {

constexpr int kFramesPerQuarter = 10;  // frames per 32 TMEM lanes
constexpr int kTileM = 128;            // GEMM rows per tile (40 frames)
constexpr int kTileFramesM = 40;
constexpr int kTileN = 128;            // GEMM columns per tile (40 frames)
constexpr int kTileFramesN = 40;
constexpr int kSliceCols = 32;         // epilogue columns per warp: one 32-row group of B
constexpr int kSliceFrames = kFramesPerQuarter;  // 10 frames (30 columns + 2 pad)
constexpr int kSlices = kTileN / kSliceCols;  // 4
constexpr int kEpiWarps = 4 * kSlices; // 16 drain warps: every (lane quarter, slice)
constexpr int kHelpWarps = 4;          // extra warps for the per-pair FP64 epilogue
constexpr int kQcpWarps = kEpiWarps + kHelpWarps;
constexpr int kTcThreads = 64 + 32 * kQcpWarps;
constexpr int kKPad = 64;              // atoms are padded to a multiple of this
constexpr int kTmemCols = 512;
constexpr int kBlockPairs = kFramesPerQuarter * kSliceFrames;  // 100 frame pairs per drain warp
// per-warp H staging, pair-major: element e = 3a + b of pair p at [e][p], so
// the epilogue's lanes (consecutive pairs) read consecutive doubles
constexpr int kEpiWarpBytes = 9 * kBlockPairs * 8;

template <int LIMBS>
struct TcGeo {
  // accumulators: shift groups kShift .. 2 LIMBS - 2 (3 limbs leave out lo x lo, group 0)
  static constexpr int kShift = LIMBS == 3 ? 1 : 0;
  static constexpr int kGroups = 2 * LIMBS - 1 - kShift;
  // atoms (= bytes per operand row) per stage: 32 with 3 limbs (4 stages of 24 KB),
  // 64 with 2 (3 stages of 32 KB); either fits 227 KB with the H staging
  static constexpr int kKChunk = LIMBS == 3 ? 32 : 64;
  static constexpr int kStages = LIMBS == 3 ? 4 : 3;
  static constexpr int kALimbBytes = kTileM * kKChunk;
  static constexpr int kBLimbBytes = kTileN * kKChunk;
  static constexpr int kABytes = LIMBS * kALimbBytes;
  static constexpr int kBBytes = LIMBS * kBLimbBytes;
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kEpiOffset = kStages * kStageBytes;
  static constexpr int kFrameOffset = kEpiOffset + kEpiWarps * kEpiWarpBytes;  // per-tile frame terms
  static constexpr int kBarOffset = kFrameOffset + 4 * (kTileFramesM + kTileFramesN) * 8;
  // full[8], empty[8], tmem_full, tmem_empty, drain, tmem address, abort flag
  static constexpr int kSmemBytes = kBarOffset + 24 * 8 + 64;
  static constexpr int kQmax = LIMBS == 3 ? (1 << 23) - (1 << 16) : (1 << 15) - (1 << 8);
  static_assert(kSmemBytes <= 227 * 1024, "shared memory");
};

// Pairs whose truncated 3-limb RMSD falls below this are recomputed exactly.
constexpr float kRefineRmsd = 0.01f;

// ------------------------------------------------------------------ PTX --

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, int ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 8 consecutive 32-bit TMEM columns -> 8 registers per thread
// (call tmem_wait_ld before using them)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// Shared-memory matrix descriptor, K-major, rows of ROW bytes with the
// matching swizzle (64: SWIZZLE_64B, layout 4; 32: SWIZZLE_32B, layout 6),
// 8-row core groups 8 ROW bytes apart, sm_100 descriptor version 1.
template <int ROW>
__device__ __forceinline__ uint64_t desc_sw(const void* p) {
  static_assert(ROW == 32 || ROW == 64, "row bytes");
  const uint64_t start = (smem_addr(p) >> 4) & 0x3FFFu;
  return start | (uint64_t(1) << 16) | (uint64_t((8 * ROW) >> 4) << 32) | (uint64_t(1) << 46) |
         (uint64_t(ROW == 64 ? 4 : 6) << 61);
}

// kind::i8 instruction descriptor: D s32, A/B s8, both K-major, M=128, N=96.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kTileN >> 3) << 17) |
                            (uint32_t(kTileM >> 4) << 24);

// bounded wait on an mbarrier phase (no shared abort fallback needed by
// callers other than through the flag)
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity, int* status, volatile int* abort,
                                        uint64_t limit_ns) {
  return mbar_wait(bar, parity, status, kStatusTimeoutFull, abort, limit_ns);
}

// Tiles are enumerated in groups of kRowGroup tile rows, column after column
// inside a group, so that the ~148 tiles in flight at once share a few A rows
// and B columns and their limbs stay in L2.  (Row after row, they would share
// one A row but stream 148 B columns, rereading each column from DRAM for
// every row once the limbs outgrow L2: 196 MB for 20,000 frames x 1,000 atoms.)
constexpr int kRowGroup = 8;

struct TileList {
  int ni, nj;  // I blocks (40 frames) x J blocks (40 frames)
  int64_t F;
  int part, parts;  // this launch computes the I blocks bi = part (mod parts)
  __device__ __forceinline__ bool valid(int64_t t, int& bi, int& bj) const {
    const int64_t gsz = (int64_t)kRowGroup * nj;
    const int64_t g = t / gsz, r = t - g * gsz;
    const int rows = min(kRowGroup, ni - (int)g * kRowGroup);
    bj = (int)(r / rows);
    bi = (int)g * kRowGroup + (int)(r - (int64_t)bj * rows);
    if (bi % parts != part) return false;
    const int64_t i0 = (int64_t)bi * kTileFramesM;
    const int64_t jmax = min((int64_t)(bj + 1) * kTileFramesN, F) - 1;
    return i0 < jmax && (int64_t)bj * kTileFramesN < F;  // some pair i < j in the tile
  }
};

struct TcArgs {
  int64_t F;
  int64_t n_pad;      // atoms padded to kKPad
  double n;           // selected atoms
  int metric;
  const double* gsum;  // [F] sum |q|^2 (units of s^2)
  const double* cen;   // [F][3] centroids (A)
  const double* scale; // device scalar s
  float* out;          // [F][F]
  int* status;
  WaitCfg wait;
  uint2* flagged;      // 3 limbs: pairs (i, j) below kRefineRmsd for pair_refine_kernel
  unsigned* n_flagged; //   their count (may exceed cap: the refine pass then scans the matrix)
  unsigned cap;
};

// -------------------------------------------------------------- kernel --

template <int LIMBS>
__global__ void __launch_bounds__(kTcThreads, 1)
    pair_tc_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                   const TcArgs args, const TileList tiles) {
  using G = TcGeo<LIMBS>;
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr int kStagesTc = G::kStages;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::kBarOffset);
  uint64_t* full = bars;
  uint64_t* empty = bars + 8;
  uint64_t* tmem_full = bars + 16;
  uint64_t* tmem_empty = tmem_full + 1;
  uint64_t* drain = tmem_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + G::kBarOffset + 24 * 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::kBarOffset + 24 * 8 + 16);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_k = (int)(args.n_pad / G::kKChunk);
  const int64_t n_tiles = (int64_t)tiles.ni * tiles.nj;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesTc; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tmem_full, 1);
    mbar_init(tmem_empty, kEpiWarps);
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      // under the error-path test CTA 0's first stage is never armed
      const bool withheld = args.wait.withhold && blockIdx.x == 0;
      uint32_t it = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        int bi, bj;
        if (!tiles.valid(t, bi, bj)) continue;
        for (int kc = 0; kc < n_k; ++kc, ++it) {
          const int s = it % kStagesTc;
          const uint32_t ph = (it / kStagesTc) & 1u;
          if (!tc_wait(&empty[s], ph ^ 1u, args.status, abort_flag, args.wait.limit_ns)) { ok = false; break; }
          if (withheld && it == 0) continue;
          unsigned char* st = smem + s * G::kStageBytes;
          mbar_arrive_expect_tx(&full[s], G::kStageBytes);
          tma_load_3d(st, &map_a, kc * G::kKChunk, bi * kTileM, 0, &full[s]);
          tma_load_3d(st + G::kABytes, &map_b, kc * G::kKChunk, bj * kTileN, 0, &full[s]);
        }
      }
      // When the MMAs stopped early (a wait ran out), stages loaded for them
      // may still be landing; every load must complete before the CTA exits.
      // In a complete run the MMAs consumed every stage and these return at once.
      const uint32_t first = it > (uint32_t)kStagesTc ? it - (uint32_t)kStagesTc : 0u;
      for (uint32_t j = first; j < it; ++j)
        if (!(withheld && j == 0)) mbar_drain(&full[j % kStagesTc], (j / kStagesTc) & 1u, args.status);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      uint32_t it = 0, tc = 0;
      bool ok = true;
      // descriptors differ only in their start-address field (address >> 4, 14
      // bits, which the shared-memory window never overflows): one base, offsets
      // added per MMA, so the issuing thread spends few instructions per MMA
      const uint64_t dbase = desc_sw<G::kKChunk>(smem);
      for (int64_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        int bi, bj;
        if (!tiles.valid(t, bi, bj)) continue;
        // the epilogue must have drained the previous tile's accumulators
        if (!tc_wait(tmem_empty, (tc & 1u) ^ 1u, args.status, abort_flag, args.wait.limit_ns)) { ok = false; break; }
        tc_fence_after();
        for (int kc = 0; kc < n_k; ++kc, ++it) {
          const int s = it % kStagesTc;
          const uint32_t ph = (it / kStagesTc) & 1u;
          if (!tc_wait(&full[s], ph, args.status, abort_flag, args.wait.limit_ns)) { ok = false; break; }
          tc_fence_after();
          const uint64_t dst = dbase + (uint64_t)((uint32_t)(s * G::kStageBytes) >> 4);
          const uint32_t later = kc > 0 ? 1u : 0u;
#pragma unroll
          for (int p = 0; p < LIMBS; ++p) {
#pragma unroll
            for (int r = 0; r < LIMBS; ++r) {
              const int g = p + r;
              if (g < G::kShift) continue;  // 3 limbs: lo x lo is left out
              // the first MMA of a group in a tile overwrites, the rest add
              const bool first_pair = (p == (g < LIMBS ? 0 : g - LIMBS + 1));
#pragma unroll
              for (int ks = 0; ks < G::kKChunk / 32; ++ks) {
                const uint64_t da = dst + (uint64_t)((p * G::kALimbBytes + ks * 32) >> 4);
                const uint64_t db = dst + (uint64_t)((G::kABytes + r * G::kBLimbBytes + ks * 32) >> 4);
                const uint32_t acc = (!first_pair || ks > 0) ? 1u : later;
                mma_i8(tmem_base + (uint32_t)((g - G::kShift) * kTileN), da, db, kIdesc, acc);
              }
            }
          }
          tc_commit(&empty[s]);  // stage free once these MMAs have read it
        }
        if (!ok) break;
        tc_commit(tmem_full);  // accumulators of this tile complete
        ++tc;
      }
      // all MMAs issued by this thread must finish before TMEM is freed
      tc_commit(drain);
      const uint64_t t0 = global_timer_ns();
      while (!mbar_try_wait(drain, 0)) {
        if (global_timer_ns() - t0 > kWaitLimitNs) {
          atomicOr(args.status, kStatusTimeoutDrain);
          break;
        }
      }
    }
  } else {
    // ---------------- epilogue ----------------
    // warps 2-13 drain TMEM (each its lane quarter x 32-column slice) into
    // shared memory; warps 14-21 stage the tile's per-frame terms; then all 20
    // run the tile's pair epilogue (QCP) two rounds deep, between two named
    // barriers (id 1 after staging, id 2 before the staging is rewritten).
    const int wq = warp - 2;       // 0..19
    const bool drainer = wq < kEpiWarps;
    const int quarter = warp & 3;  // TMEM lane quarter a drain warp may access
    const int slice = wq >> 2;     // 32-column slice (10 frames) of a drain warp
    const double s = *args.scale;
    const double s2 = s * s;
    const float s2f = (float)s2;
    const float nf = (float)args.n;
    // per-frame terms [4][80]: G (units of s^2), then centroids cx, cy, cz
    double* frm = reinterpret_cast<double*>(smem + G::kFrameOffset);
    constexpr int kTf = kTileFramesM + kTileFramesN;
    uint32_t tc = 0;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
      int bi, bj;
      if (!tiles.valid(t, bi, bj)) continue;
      if (drainer) {
        if (tc_wait(tmem_full, tc & 1u, args.status, abort_flag, args.wait.limit_ns)) {
          tc_fence_after();
          long long* epi = reinterpret_cast<long long*>(smem + G::kEpiOffset + wq * kEpiWarpBytes);
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            // columns [16 half, 16 half + 16) of the slice; 30 are frame columns
            long long acc[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) acc[c] = 0;
#pragma unroll
            for (int g = 0; g < G::kGroups; ++g) {
              int32_t v[16];
              const uint32_t col = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                                   (uint32_t)(g * kTileN + slice * kSliceCols + 16 * half);
              tmem_ld8(col, v);
              tmem_ld8(col + 8, v + 8);
              tmem_wait_ld();
#pragma unroll
              for (int c = 0; c < 16; ++c) acc[c] += (long long)v[c] << (8 * (g + G::kShift));
            }
            if (lane < 30) {
              // lane = 3 pi + a (row frame pi, component a); column 3 pj + b
              const int pi = lane / 3, a = lane - 3 * pi;
              long long* row = epi + a * 3 * kBlockPairs + pi * kSliceFrames;
#pragma unroll
              for (int c = 0; c < 16; ++c) {
                const int cc = 16 * half + c;
                if (cc < 30) row[(cc % 3) * kBlockPairs + cc / 3] = acc[c];  // exact, units of s^2
              }
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(tmem_empty);  // MMAs of the next tile may start
        }
      } else {
        // per-frame terms of the tile's 40 row frames and 30 column frames
        for (int q = (wq - kEpiWarps) * 32 + lane; q < kTf; q += kHelpWarps * 32) {
          const int64_t f = q < kTileFramesM ? (int64_t)bi * kTileFramesM + q
                                             : (int64_t)bj * kTileFramesN + (q - kTileFramesM);
          const bool in = f < args.F;
          frm[q] = in ? args.gsum[f] : 0.0;
          frm[kTf + q] = in ? args.cen[f * 3 + 0] : 0.0;
          frm[2 * kTf + q] = in ? args.cen[f * 3 + 1] : 0.0;
          frm[3 * kTf + q] = in ? args.cen[f * 3 + 2] : 0.0;
        }
      }
      ++tc;
      named_barrier_sync(1, 32 * kQcpWarps);
      if (*abort_flag) break;
      // 12 blocks x 100 pairs, two rounds of 20 warps x 32 lanes
      constexpr int kPairs = kEpiWarps * kFramesPerQuarter * kSliceFrames;  // 1200
#pragma unroll 1
      for (int gp = wq * 32 + lane; gp < kPairs; gp += kQcpWarps * 32) {
        const int blk = gp / kBlockPairs, pl = gp - blk * kBlockPairs;
        const int pi = pl / kSliceFrames, pj = pl - pi * kSliceFrames;
        const int bq = (blk + 2) & 3, bs = blk >> 2;  // lane quarter and slice of drain warp blk
        const int fi = bq * kFramesPerQuarter + pi, fj = kTileFramesM + bs * kSliceFrames + pj;
        const int64_t i = (int64_t)bi * kTileFramesM + fi - 0;
        const int64_t j = (int64_t)bj * kTileFramesN + bs * kSliceFrames + pj;
        if (!(i < j && j < args.F)) continue;
        const long long* epi = reinterpret_cast<const long long*>(smem + G::kEpiOffset + blk * kEpiWarpBytes);
        long long h[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) h[e] = epi[e * kBlockPairs + pl];
        const double gi = frm[fi], gj = frm[fj];
        float v;
        if (args.metric == WMD_PAIR_NOFIT) {
          // sum |q_i - q_j|^2 = G_i + G_j - 2 tr H (exact inputs, double-float), plus n |c_i - c_j|^2
          const double dq = gi + gj - 2.0 * ((double)h[0] + (double)h[4] + (double)h[8]);
          const float d0 = (float)(frm[kTf + fi] - frm[kTf + fj]);
          const float d1 = (float)(frm[2 * kTf + fi] - frm[2 * kTf + fj]);
          const float d2 = (float)(frm[3 * kTf + fi] - frm[3 * kTf + fj]);
          const float ssq = (float)dq * s2f + nf * (d0 * d0 + d1 * d1 + d2 * d2);
          v = ssq > 0.0f ? sqrtf(ssq / nf) : 0.0f;
        } else {
          float msd;
          if (!qcp_msd_mixed(h, gi, gj, nf, s2f, &msd)) {  // a root that is not simple: the FP64 route
            double hd[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) hd[e] = (double)h[e] * s2;
            const double gid = gi * s2, gjd = gj * s2;
            const QcpOut q = qcp_lambda(hd, 0.5 * (gid + gjd));
            msd = (float)msd_from(gid, gjd, q.lambda, args.n);
          }
          v = sqrtf(msd);
        }
        args.out[(size_t)i * args.F + j] = v;
        args.out[(size_t)j * args.F + i] = v;
        if (G::kShift && v < kRefineRmsd) {  // recomputed exactly by pair_refine_kernel
          const unsigned k = atomicAdd(args.n_flagged, 1u);
          if (k < args.cap) args.flagged[k] = make_uint2((unsigned)i, (unsigned)j);
        }
      }
      named_barrier_sync(2, 32 * kQcpWarps);  // staging may be rewritten
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
}

// --------------------------------------------------------------- prep --

// Pass 1 (one CTA per frame): FP64 centroid and max |x - c| over the frame,
// folded into a global maximum (non-negative floats compare as unsigned).
__global__ void __launch_bounds__(256) tc_prep_centre(const float* __restrict__ coords, int64_t n_atoms, int stride,
                                                      const uint32_t* __restrict__ sel, int64_t n_sel,
                                                      double* __restrict__ cen, unsigned* __restrict__ maxbits,
                                                      int* status) {
  __shared__ double red[8][3];
  __shared__ float mred[8];
  const int64_t f = blockIdx.x;
  const float* fr = coords + (size_t)f * n_atoms * stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
    int64_t idx = sel ? (int64_t)sel[k] : k;
    if (idx >= n_atoms) {
      atomicOr(status, kStatusBadIndex);
      idx = 0;
    }
    const float* p = fr + idx * stride;
    s0 += p[0]; s1 += p[1]; s2 += p[2];
  }
  for (int o = 16; o; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) { red[warp][0] = s0; red[warp][1] = s1; red[warp][2] = s2; }
  __syncthreads();
  double c[3] = {0, 0, 0};
  for (int w = 0; w < 8; ++w) { c[0] += red[w][0]; c[1] += red[w][1]; c[2] += red[w][2]; }
  const double inv = 1.0 / (double)n_sel;
  c[0] *= inv; c[1] *= inv; c[2] *= inv;
  float m = 0.f;
  for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
    int64_t idx = sel ? (int64_t)sel[k] : k;
    if (idx >= n_atoms) idx = 0;
    const float* p = fr + idx * stride;
    for (int q = 0; q < 3; ++q) m = fmaxf(m, (float)fabs((double)p[q] - c[q]));
  }
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) mred[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float mm = 0.f;
    for (int w = 0; w < 8; ++w) mm = fmaxf(mm, mred[w]);
    atomicMax(maxbits, __float_as_uint(mm));
    cen[f * 3 + 0] = c[0]; cen[f * 3 + 1] = c[1]; cen[f * 3 + 2] = c[2];
  }
}

// Pass 2 (one CTA per frame): quantise with the trajectory-wide scale and
// write the int8 limbs L[p][row(f, a)][k]; G_f = sum q^2 exactly (int64),
// less sum lo^2 with 3 limbs (the products the tensor cores form).
template <int LIMBS>
__global__ void __launch_bounds__(256) tc_prep_limbs(const float* __restrict__ coords, int64_t n_atoms, int stride,
                                                     const uint32_t* __restrict__ sel, int64_t n_sel, int64_t n_pad,
                                                     int64_t rows, const double* __restrict__ cen,
                                                     const unsigned* __restrict__ maxbits,
                                                     int8_t* __restrict__ limbs, double* __restrict__ gsum,
                                                     double* __restrict__ scale_out) {
  __shared__ long long red[8];
  constexpr int qmax = TcGeo<LIMBS>::kQmax;
  const int64_t f = blockIdx.x;
  const float mx = __uint_as_float(*maxbits);
  const double s = mx > 0.f ? (double)mx / (double)qmax * (1.0 + 1e-12) : 1.0;
  if (f == 0 && threadIdx.x == 0) *scale_out = s;
  const double inv_s = 1.0 / s;
  const float* fr = coords + (size_t)f * n_atoms * stride;
  const double c[3] = {cen[f * 3 + 0], cen[f * 3 + 1], cen[f * 3 + 2]};
  const int64_t row0 = (f / kFramesPerQuarter) * 32 + (f % kFramesPerQuarter) * 3;
  long long g = 0;
  for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
    int64_t idx = sel ? (int64_t)sel[k] : k;
    if (idx >= n_atoms) idx = 0;
    const float* p = fr + idx * stride;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      long long q = llrint(((double)p[a] - c[a]) * inv_s);
      q = q > qmax ? qmax : (q < -qmax ? -qmax : q);
      g += q * q;
      int32_t rem = (int32_t)q;
#pragma unroll
      for (int l = 0; l < LIMBS; ++l) {
        // balanced base-256 digit in [-128, 127]
        int32_t d = ((rem % 256) + 256 + 128) % 256 - 128;
        if (l == LIMBS - 1) d = rem;
        // the self-sum G leaves out lo x lo as the tensor-core products do
        if (l == 0 && TcGeo<LIMBS>::kShift) g -= (long long)d * d;
        limbs[((size_t)l * rows + row0 + a) * n_pad + k] = (int8_t)d;
        rem = (rem - d) / 256;
      }
    }
  }
  for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = g;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < 8; ++w) t += red[w];
    gsum[f] = (double)t;
  }
}

// 3 limbs: pairs whose truncated RMSD came out below kRefineRmsd, recomputed
// exactly in FP64 from the coordinates, a warp per pair: the centred sums H,
// G_i, G_j and QCP (metric rms), or sum |x_i - x_j|^2 (nofit), each lane
// taking atoms lane, lane + 32, ... and the warp adding its lanes in a fixed
// tree.  When more pairs were flagged than the list holds, every pair (i, j),
// i < j, of this launch's tile rows (i / 40 = part mod parts) whose entry is
// below kRefineRmsd is found in the matrix itself.
__global__ void __launch_bounds__(256) pair_refine_kernel(const float* __restrict__ coords, int64_t n_atoms, int stride,
                                                          const uint32_t* __restrict__ sel, int64_t n_sel, int64_t F,
                                                          const double* __restrict__ cen, int metric,
                                                          const uint2* __restrict__ list,
                                                          const unsigned* __restrict__ count, unsigned cap,
                                                          float* __restrict__ out, int part, int parts, int* status) {
  const int lane = threadIdx.x & 31;
  const int64_t wg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned n_list = *count;
  auto refine = [&](int64_t i, int64_t j) {
    const float* xi = coords + (size_t)i * n_atoms * stride;
    const float* xj = coords + (size_t)j * n_atoms * stride;
    const double ci0 = cen[i * 3], ci1 = cen[i * 3 + 1], ci2 = cen[i * 3 + 2];
    const double cj0 = cen[j * 3], cj1 = cen[j * 3 + 1], cj2 = cen[j * 3 + 2];
    double v[12];
#pragma unroll
    for (int e = 0; e < 12; ++e) v[e] = 0.0;
    for (int64_t k = lane; k < n_sel; k += 32) {
      int64_t a = sel ? (int64_t)sel[k] : k;
      if (a >= n_atoms) {  // bad device-side selection: report, read atom 0
        atomicOr(status, kStatusBadIndex);
        a = 0;
      }
      const float* p = xi + a * stride;
      const float* q = xj + a * stride;
      if (metric == WMD_PAIR_NOFIT) {
        const double d0 = (double)p[0] - (double)q[0], d1 = (double)p[1] - (double)q[1],
                     d2 = (double)p[2] - (double)q[2];
        v[0] += d0 * d0 + d1 * d1 + d2 * d2;
      } else {
        const double u0 = (double)p[0] - ci0, u1 = (double)p[1] - ci1, u2 = (double)p[2] - ci2;
        const double w0 = (double)q[0] - cj0, w1 = (double)q[1] - cj1, w2 = (double)q[2] - cj2;
        v[0] += u0 * w0; v[1] += u0 * w1; v[2] += u0 * w2;
        v[3] += u1 * w0; v[4] += u1 * w1; v[5] += u1 * w2;
        v[6] += u2 * w0; v[7] += u2 * w1; v[8] += u2 * w2;
        v[9] += u0 * u0 + u1 * u1 + u2 * u2;
        v[10] += w0 * w0 + w1 * w1 + w2 * w2;
      }
    }
#pragma unroll
    for (int e = 0; e < 11; ++e)
      for (int o = 16; o; o >>= 1) v[e] += __shfl_xor_sync(0xffffffffu, v[e], o);
    if (lane == 0) {
      const double nn = (double)n_sel;
      double r;
      if (metric == WMD_PAIR_NOFIT) {
        r = sqrt(v[0] / nn);
      } else {
        const QcpOut qo = qcp_lambda(v, 0.5 * (v[9] + v[10]));
        r = sqrt(msd_from(v[9], v[10], qo.lambda, nn));
      }
      out[(size_t)i * F + j] = (float)r;
      out[(size_t)j * F + i] = (float)r;
    }
  };
  if (n_list <= cap) {
    for (int64_t p = wg; p < (int64_t)n_list; p += nw) refine(list[p].x, list[p].y);
    return;
  }
  for (int64_t i = wg; i < F; i += nw) {
    if ((int)((i / kTileFramesM) % parts) != part) continue;
    for (int64_t j0 = i + 1; j0 < F; j0 += 32) {
      const int64_t j = j0 + lane;
      const bool low = j < F && out[(size_t)i * F + j] < kRefineRmsd;
      unsigned m = __ballot_sync(0xffffffffu, low);
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        refine(i, j0 + b);
      }
    }
  }
}

// ---------------------------------------------------------------- host --

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn(std::string* msg) {
  static EncodeTiled fn = nullptr;
  if (fn) return fn;
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    *msg = "cuda driver error: cuTensorMapEncodeTiled unavailable";
    return nullptr;
  }
  fn = reinterpret_cast<EncodeTiled>(p);
  return fn;
}

template <int LIMBS>
int run_tc(PairwiseWorkspace& w, int sm_count, const float* coords, int64_t F, int64_t n_atoms, int stride,
           const uint32_t* sel, int64_t n_sel, int metric, float* out, int* status, const WaitCfg& wait,
           cudaStream_t s, std::string* msg) {
  using G = TcGeo<LIMBS>;
  const int64_t n_pad = (n_sel + kKPad - 1) / kKPad * kKPad;
  const int64_t rows = (F + kFramesPerQuarter - 1) / kFramesPerQuarter * 32;
  const int64_t rows_pad = (rows + kTileM - 1) / kTileM * kTileM;  // whole 128-row tiles
  const size_t limb_bytes = (size_t)LIMBS * rows_pad * n_pad;
  const size_t small = 256 + (size_t)F * (sizeof(double) * 4);
  // pairs flagged for the exact recomputation (3 limbs)
  const unsigned cap = G::kShift ? (unsigned)std::min<int64_t>(std::max<int64_t>(F * (F - 1) / 2, 1), 1 << 20) : 0u;
  const size_t list_bytes = (size_t)cap * sizeof(uint2);
  // workspace: [scale, maxbits, flagged count | gsum F | cen 3F][limbs][flagged pairs]
  const size_t need = small + limb_bytes + 1024 + list_bytes + 16;
  if (!w.extra || w.extra_bytes < need) {
    if (w.extra) cudaFree(w.extra);
    w.extra = nullptr;
    w.extra_bytes = 0;
    cudaError_t e = cudaMalloc(&w.extra, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *msg = std::string("cuda driver error: pairwise workspace allocation failed: ") + cudaGetErrorString(e);
      return WMD_ERR_OOM;
    }
    w.extra_bytes = need;
  }
  unsigned char* base = static_cast<unsigned char*>(w.extra);
  double* scale = reinterpret_cast<double*>(base);
  unsigned* maxbits = reinterpret_cast<unsigned*>(base + 8);
  double* gsum = reinterpret_cast<double*>(base + 256);
  double* cen = gsum + F;
  unsigned* n_flagged = reinterpret_cast<unsigned*>(base + 16);
  int8_t* limbs = reinterpret_cast<int8_t*>(base + ((small + 1023) & ~size_t(1023)));
  uint2* flagged = reinterpret_cast<uint2*>(base + (((small + 1023) & ~size_t(1023)) + limb_bytes + 15) / 16 * 16);

  cudaError_t e = cudaMemsetAsync(base, 0, 256, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(limbs, 0, limb_bytes, s);
  if (e != cudaSuccess) {
    *msg = std::string("cuda driver error: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  tc_prep_centre<<<(unsigned)F, 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, cen, maxbits, status);
  tc_prep_limbs<LIMBS><<<(unsigned)F, 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, n_pad, rows_pad, cen, maxbits,
                                                   limbs, gsum, scale);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    *msg = std::string("cuda driver error: pairwise prep: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }

  EncodeTiled enc = encode_fn(msg);
  if (!enc) return WMD_ERR_CUDA;
  CUtensorMap map_a, map_b;
  const cuuint64_t dims[3] = {(cuuint64_t)n_pad, (cuuint64_t)rows_pad, (cuuint64_t)LIMBS};
  const cuuint64_t strides[2] = {(cuuint64_t)n_pad, (cuuint64_t)(rows_pad * n_pad)};
  const cuuint32_t box_a[3] = {G::kKChunk, kTileM, LIMBS};
  const cuuint32_t box_b[3] = {G::kKChunk, kTileN, LIMBS};
  const CUtensorMapSwizzle swz = G::kKChunk == 32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B;
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(&map_a, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, limbs, dims, strides, box_a, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r == CUDA_SUCCESS)
    r = enc(&map_b, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, limbs, dims, strides, box_b, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    *msg = "cuda driver error: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return WMD_ERR_CUDA;
  }

  TcArgs a;
  a.F = F;
  a.n_pad = n_pad;
  a.n = (double)n_sel;
  a.metric = metric;
  a.gsum = gsum;
  a.cen = cen;
  a.scale = scale;
  a.out = out;
  a.status = status;
  a.wait = wait;
  a.flagged = flagged;
  a.n_flagged = n_flagged;
  a.cap = cap;
  TileList tl;
  tl.ni = (int)((F + kTileFramesM - 1) / kTileFramesM);
  tl.nj = (int)((F + kTileFramesN - 1) / kTileFramesN);
  tl.F = F;
  tl.part = w.part;
  tl.parts = w.parts;
  auto kern = pair_tc_kernel<LIMBS>;
  if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmemBytes)) != cudaSuccess) {
    *msg = std::string("cuda driver error: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  const int64_t n_tiles = (int64_t)tl.ni * tl.nj;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(sm_count, n_tiles));
  kern<<<grid, kTcThreads, G::kSmemBytes, s>>>(map_a, map_b, a, tl);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    *msg = std::string("cuda driver error: pairwise tensor-core launch: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  if (G::kShift) {
    pair_refine_kernel<<<(unsigned)(2 * sm_count), 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, F, cen, metric,
                                                                 flagged, n_flagged, cap, out, w.part, w.parts, status);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      *msg = std::string("cuda driver error: pairwise refine launch: ") + cudaGetErrorString(e);
      return WMD_ERR_CUDA;
    }
  }
  return 0;
}

}  // namespace

int pairwise_tc_run(PairwiseWorkspace& w, int sm_count, const float* coords, int64_t n_frames, int64_t n_atoms,
                    int stride, const uint32_t* sel, int64_t n_sel, int metric, int limbs, float* out, int* status,
                    const WaitCfg& wait, cudaStream_t s, std::string* msg) {
  // exact int32 accumulation: LIMBS n_pad 128^2 < 2^31
  const int64_t max_atoms = limbs == 3 ? 43648 : 65472;
  if (n_sel > max_atoms) {
    *msg = "tensor-core pairwise modes accept at most " + std::to_string(max_atoms) +
           " selected atoms (exact int32 accumulation); use WMD_MODE_FP64";
    return WMD_ERR_UNSUPPORTED;
  }
  if (n_frames > (int64_t)1 << 31) {
    *msg = "too many frames for one pairwise call";
    return WMD_ERR_INVALID_ARG;
  }
  return limbs == 3
             ? run_tc<3>(w, sm_count, coords, n_frames, n_atoms, stride, sel, n_sel, metric, out, status, wait, s, msg)
             : run_tc<2>(w, sm_count, coords, n_frames, n_atoms, stride, sel, n_sel, metric, out, status, wait, s, msg);
}

}  // namespace wmd

// rmsd_lanes.cu -- per-frame RMSD statistics with frames across lanes.
//
// The atom-major streaming kernel (rmsd_frames.cu) gives every thread a few
// atoms of one frame, so each (tile, frame) item ends in a 15-value
// cross-lane reduction and a CTA barrier; those cost about as many
// instructions as the FP64 arithmetic itself.  Here the roles are swapped:
//
//   * A warp owns a run of stages; a stage is 32 frames x 32 atoms (lane l =
//     frame 32g + l).  The frames' coordinates arrive by 2-D TMA (boxes of 32
//     rows x 128 bytes, 128-byte swizzle, so that every lane reading "its"
//     row hits a different bank group), the 32 reference atoms (centred,
//     FP64) by a 1-D bulk copy next to them.  Two stages per warp, refilled
//     by lane 0 as soon as the warp is done with one.
//   * Each lane adds, in FP64 and in atom order, the 15 sums of its own frame
//     (sum x, sum x_a^2, sum x y_c^T): no shuffles, no barriers.
//   * Atoms are grouped into tiles (256 to 2,048 atoms, chosen per launch so
//     that whole units balance over the warp slots); a unit is (tile,
//     32-frame group) and belongs to one warp, which stores each lane's 16 sums into
//     the same [frame][tile][16] partials the finalize kernel reads.  Every
//     warp gets the same number of whole units, so results do not depend on
//     the launch shape and are bitwise reproducible.
//
// Frames whose stride is not a multiple of 16 bytes (packed xyz with
// n_atoms % 4 != 0) cannot be rows of a tensor map; four consecutive frames
// can (48 n_atoms bytes).  Such launches (dense selections) read "quad rows":
// a stage is four boxes of [8 quad rows x 100 floats], box j holding frames
// 32g + 4i + j (i = 0..7).  Box j starts at the 16-byte boundary at or below
// frame position j's first atom of the stage, so lane 4i + j reads its 96
// floats at a fixed offset of (3 j n_atoms) mod 4 floats with 32-bit loads:
// rows of 400 bytes put the 32 lanes in distinct banks for odd n_atoms (two
// lanes per bank otherwise).  Atoms past the tile come from the next frame of
// the quad row and are masked.  The last n_frames mod 4 frames are left to the
// gathered kernel, with the same tiles and partial layout.
//
// Atoms streamed: a dense selection (the first n_sel atoms), or the span
// [lane_atom0, lane_atom0 + lane_atoms) of a sorted selection with the
// reference expanded onto it and per-atom weights (1 for selected atoms, 0
// for the rest; or the masses of a weighted reference).  The weights also
// serve weighted references over dense selections.  Requirements (else the
// atom-major kernel runs): a 16-byte aligned first streamed atom and a frame
// stride that is a multiple of 16 bytes (n_atoms % 4 == 0 for packed xyz).
// The reference values and weights must be padded with 32 zero atoms (the
// bulk copies of the last stage read past the span).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "device_util.cuh"
#include "wmd_internal.h"

namespace wmd {

namespace {

constexpr int kLaneWarps = 4;   // warps per CTA
constexpr int kLaneStages = 2;  // stage ring per warp
constexpr int kLaneAtoms = 32;  // atoms per stage

template <int STRIDE>
struct LaneGeo {
  static constexpr int kBoxes = kLaneAtoms * STRIDE / 32;  // [32 frames][32 floats] boxes per stage
  static constexpr int kXBytes = kBoxes * 32 * 32 * 4;
  static constexpr int kYBytes = kLaneAtoms * 3 * 8;
  static constexpr int kWBytes = kLaneAtoms * 4;  // per-atom weights (weighted / expanded launches)
  static constexpr int kStageBytes = (kXBytes + kYBytes + kWBytes + 1023) / 1024 * 1024;
  static constexpr int kBarOffset = kLaneWarps * kLaneStages * kStageBytes;
  static constexpr int kAbortOffset = kBarOffset + kLaneWarps * kLaneStages * 8;
  static constexpr int kSmemBytes = kAbortOffset + 16 + 1024;  // + slack to align the base to 1024
};

// quad rows (packed xyz, n_atoms % 4 != 0): 4 boxes of [8 quad rows x 100 floats], no swizzle
struct QuadGeo {
  static constexpr int kBoxRowBytes = 100 * 4;
  static constexpr int kBoxBytes = 8 * kBoxRowBytes;
  static constexpr int kXBytes = 4 * kBoxBytes;
  static constexpr int kYBytes = kLaneAtoms * 3 * 8;
  static constexpr int kWBytes = kLaneAtoms * 4;
  static constexpr int kStageBytes = (kXBytes + kYBytes + kWBytes + 127) / 128 * 128;
  static constexpr int kBarOffset = kLaneWarps * kLaneStages * kStageBytes;
  static constexpr int kAbortOffset = kBarOffset + kLaneWarps * kLaneStages * 8;
  static constexpr int kSmemBytes = kAbortOffset + 16 + 1024;
};

template <bool QUAD, int STRIDE>
struct PickGeo {
  using type = LaneGeo<STRIDE>;
};
template <int STRIDE>
struct PickGeo<true, STRIDE> {
  using type = QuadGeo;
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// One lane's sums over the valid atoms of a stage (valid is warp-uniform).
// Packed xyz: 4 atoms = 3 swizzled 16-byte chunks; xyzw: 1 atom = 1 chunk.
template <int STRIDE, bool RAW, bool W>
__device__ __forceinline__ void stage_sums(double (&acc)[15], const unsigned char* st, int lane, int valid,
                                           const FrameLaunch& L) {
  const float* wb = reinterpret_cast<const float*>(st + LaneGeo<STRIDE>::kXBytes + LaneGeo<STRIDE>::kYBytes);
  const unsigned char* row = st + lane * 128;
  const int sw = lane & 7;
  auto chunk = [&](int c) -> float4 {
    return *reinterpret_cast<const float4*>(row + (c >> 3) * 4096 + (((c & 7) ^ sw) << 4));
  };
  const double2* yb = reinterpret_cast<const double2*>(st + LaneGeo<STRIDE>::kXBytes);
  // k: the atom's index within the stage (its weight; y is pre-multiplied)
  auto add_atom = [&](float fx, float fy, float fz, double y0, double y1, double y2, bool in, int k) {
    const double x0 = fx, x1 = fy, x2 = fz;
    if (W && RAW) in = in && wb[k] != 0.0f;  // expanded selection: unselected atoms have weight 0
    if (RAW) {
      const double d0 = x0 - (y0 + L.ref.mean[0]);
      const double d1 = x1 - (y1 + L.ref.mean[1]);
      const double d2 = x2 - (y2 + L.ref.mean[2]);
      acc[0] = fma(d0, in ? d0 : 0.0, acc[0]);
      acc[1] = fma(d1, in ? d1 : 0.0, acc[1]);
      acc[2] = fma(d2, in ? d2 : 0.0, acc[2]);
    } else {
      if (W) {  // sum w x, sum w x_a^2 (the weighted forms of rmsd_frames_kernel)
        const double w = wb[k];
        const double u0 = w * x0, u1 = w * x1, u2 = w * x2;
        acc[0] += u0; acc[1] += u1; acc[2] += u2;
        acc[3] = fma(u0, x0, acc[3]); acc[4] = fma(u1, x1, acc[4]); acc[5] = fma(u2, x2, acc[5]);
      } else {
        acc[0] += x0; acc[1] += x1; acc[2] += x2;
        acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
      }
      acc[6] = fma(x0, y0, acc[6]);  acc[7] = fma(x0, y1, acc[7]);  acc[8] = fma(x0, y2, acc[8]);
      acc[9] = fma(x1, y0, acc[9]);  acc[10] = fma(x1, y1, acc[10]); acc[11] = fma(x1, y2, acc[11]);
      acc[12] = fma(x2, y0, acc[12]); acc[13] = fma(x2, y1, acc[13]); acc[14] = fma(x2, y2, acc[14]);
    }
  };
  if (STRIDE == 3) {
#pragma unroll
    for (int m = 0; m < kLaneAtoms / 4; ++m) {
      if (4 * m >= valid) break;
      const float4 a = chunk(3 * m), b = chunk(3 * m + 1), c = chunk(3 * m + 2);
      const double2 y01 = yb[6 * m + 0], y23 = yb[6 * m + 1], y45 = yb[6 * m + 2];
      const double2 y67 = yb[6 * m + 3], y89 = yb[6 * m + 4], yab = yb[6 * m + 5];
      add_atom(a.x, a.y, a.z, y01.x, y01.y, y23.x, 4 * m + 0 < valid, 4 * m + 0);
      add_atom(a.w, b.x, b.y, y23.y, y45.x, y45.y, 4 * m + 1 < valid, 4 * m + 1);
      add_atom(b.z, b.w, c.x, y67.x, y67.y, y89.x, 4 * m + 2 < valid, 4 * m + 2);
      add_atom(c.y, c.z, c.w, y89.y, yab.x, yab.y, 4 * m + 3 < valid, 4 * m + 3);
    }
  } else {
#pragma unroll
    for (int m = 0; m < kLaneAtoms / 2; ++m) {
      if (2 * m >= valid) break;
      const float4 a = chunk(2 * m), b = chunk(2 * m + 1);
      const double2 y01 = yb[3 * m + 0], y23 = yb[3 * m + 1], y45 = yb[3 * m + 2];
      add_atom(a.x, a.y, a.z, y01.x, y01.y, y23.x, 2 * m + 0 < valid, 2 * m + 0);
      add_atom(b.x, b.y, b.z, y23.y, y45.x, y45.y, 2 * m + 1 < valid, 2 * m + 1);
    }
  }
}

// The quad-row form of stage_sums: lane 4i + j reads frame position j's box,
// row i, from float offset off; atoms at or past `valid` are masked.
template <bool RAW, bool W>
__device__ __forceinline__ void stage_sums_quad(double (&acc)[15], const unsigned char* st, int lane, int off,
                                                int valid, const FrameLaunch& L) {
  const float* wb = reinterpret_cast<const float*>(st + QuadGeo::kXBytes + QuadGeo::kYBytes);
  const float* row =
      reinterpret_cast<const float*>(st + (lane & 3) * QuadGeo::kBoxBytes + (lane >> 2) * QuadGeo::kBoxRowBytes) + off;
  const double* yb = reinterpret_cast<const double*>(st + QuadGeo::kXBytes);
#pragma unroll 4
  for (int k = 0; k < kLaneAtoms; ++k) {
    if (k >= valid) break;
    const double x0 = row[3 * k], x1 = row[3 * k + 1], x2 = row[3 * k + 2];
    const double y0 = yb[3 * k], y1 = yb[3 * k + 1], y2 = yb[3 * k + 2];
    if (RAW) {
      const bool in = !W || wb[k] != 0.0f;
      const double d0 = x0 - (y0 + L.ref.mean[0]);
      const double d1 = x1 - (y1 + L.ref.mean[1]);
      const double d2 = x2 - (y2 + L.ref.mean[2]);
      acc[0] = fma(d0, in ? d0 : 0.0, acc[0]);
      acc[1] = fma(d1, in ? d1 : 0.0, acc[1]);
      acc[2] = fma(d2, in ? d2 : 0.0, acc[2]);
    } else {
      if (W) {
        const double w = wb[k];
        const double u0 = w * x0, u1 = w * x1, u2 = w * x2;
        acc[0] += u0; acc[1] += u1; acc[2] += u2;
        acc[3] = fma(u0, x0, acc[3]); acc[4] = fma(u1, x1, acc[4]); acc[5] = fma(u2, x2, acc[5]);
      } else {
        acc[0] += x0; acc[1] += x1; acc[2] += x2;
        acc[3] = fma(x0, x0, acc[3]); acc[4] = fma(x1, x1, acc[4]); acc[5] = fma(x2, x2, acc[5]);
      }
      acc[6] = fma(x0, y0, acc[6]);  acc[7] = fma(x0, y1, acc[7]);  acc[8] = fma(x0, y2, acc[8]);
      acc[9] = fma(x1, y0, acc[9]);  acc[10] = fma(x1, y1, acc[10]); acc[11] = fma(x1, y2, acc[11]);
      acc[12] = fma(x2, y0, acc[12]); acc[13] = fma(x2, y1, acc[13]); acc[14] = fma(x2, y2, acc[14]);
    }
  }
}

template <int STRIDE, bool RAW, bool W, bool QUAD = false>
__global__ void __launch_bounds__(kLaneWarps * 32) rmsd_lanes_kernel(const __grid_constant__ CUtensorMap map,
                                                                     const FrameLaunch L) {
  using G = typename PickGeo<QUAD, STRIDE>::type;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + G::kBarOffset);
  uint64_t* full = bars + warp * kLaneStages;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + G::kAbortOffset);
  unsigned char* ring = smem + warp * kLaneStages * G::kStageBytes;

  // atoms streamed: the selection itself, or the atom span an expanded
  // selection covers (L.lane_atom0 is folded into the tensor map's base)
  const int64_t F = L.n_frames, n_sel = L.lane_atoms;
  const int64_t groups = (F + 31) / 32;
  const int64_t tile = L.tile_atoms;  // a multiple of kLaneAtoms
  const int n_tiles = (int)((n_sel + tile - 1) / tile);
  const int64_t units = groups * n_tiles;  // (tile, frame group), tile-major
  const int64_t nw = L.lane_warps, gw = (int64_t)blockIdx.x * kLaneWarps + warp;
  const int64_t u0 = units * gw / nw, u1 = units * (gw + 1) / nw;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kLaneWarps * kLaneStages; ++i) mbar_init(&bars[i], 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (gw >= nw || u0 >= u1) return;

  auto unit_stages = [&](int64_t u) {
    const int64_t t = u / groups;
    return (int)((min(tile, n_sel - t * tile) + kLaneAtoms - 1) / kLaneAtoms);
  };
  // producer cursor (lane 0): unit pu, stage pk; n_issued stages so far
  int64_t pu = u0;
  int pk = 0, p_kst = unit_stages(u0);
  int64_t n_issued = 0;
  // under the error-path test the first stage of CTA 0's warp 0 is never armed
  const bool withheld = L.wait.withhold && blockIdx.x == 0 && warp == 0;
  auto issue_next = [&]() {  // lane 0
    const int64_t t = pu / groups, g = pu - t * groups;
    const int slot = (int)(n_issued % kLaneStages);
    unsigned char* dst = ring + slot * G::kStageBytes;
    const int64_t a0 = t * tile + (int64_t)pk * kLaneAtoms;
    if (!(withheld && n_issued == 0)) {
      // the warp's earlier generic reads of this slot before the async writes
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&full[slot], G::kXBytes + G::kYBytes + (W ? G::kWBytes : 0));
      if (QUAD) {
        // frame position j of the quad rows 8g .. 8g + 7: its atoms a0 .. a0 + 31
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int64_t e = (int64_t)j * 3 * L.n_atoms + 3 * a0;
          tma_load_2d(dst + j * QuadGeo::kBoxBytes, &map, (int)(e & ~int64_t(3)), (int)(g * 8), &full[slot]);
        }
      } else {
#pragma unroll
        for (int b = 0; b < LaneGeo<STRIDE>::kBoxes; ++b)
          tma_load_2d(dst + b * 4096, &map, (int)(a0 * STRIDE + 32 * b), (int)(g * 32), &full[slot]);
      }
      bulk_copy_g2s(dst + G::kXBytes, L.lane_y + a0 * 3, G::kYBytes, &full[slot]);
      if (W) bulk_copy_g2s(dst + G::kXBytes + G::kYBytes, L.lane_w + a0, G::kWBytes, &full[slot]);
    }
    ++n_issued;
    if (++pk == p_kst && ++pu < u1) {
      pk = 0;
      p_kst = unit_stages(pu);
    }
  };
  if (lane == 0)
    while (n_issued < kLaneStages && pu < u1) issue_next();

  // quad rows: this lane's float offset into its box row (stages start at
  // multiples of 32 atoms, so only the frame position matters)
  const int quad_off = QUAD ? (int)(((int64_t)(lane & 3) * 3 * L.n_atoms) & 3) : 0;
  int64_t n_done = 0;
  bool aborted = false;
  for (int64_t u = u0; u < u1 && !aborted; ++u) {
    const int64_t t = u / groups, g = u - t * groups;
    const int kst = unit_stages(u);
    double acc[15];
#pragma unroll
    for (int e = 0; e < 15; ++e) acc[e] = 0.0;
    for (int k = 0; k < kst; ++k) {
      const int slot = (int)(n_done % kLaneStages);
      const uint32_t parity = (uint32_t)((n_done / kLaneStages) & 1);
      if (!mbar_wait(&full[slot], parity, L.status, kStatusTimeoutFull, abort_flag, L.wait.limit_ns)) {
        aborted = true;
        break;
      }
      const int64_t a0 = t * tile + (int64_t)k * kLaneAtoms;
      const int valid = (int)min((int64_t)kLaneAtoms, n_sel - a0);
      if (QUAD)
        stage_sums_quad<RAW, W>(acc, ring + slot * G::kStageBytes, lane, quad_off, valid, L);
      else
        stage_sums<STRIDE, RAW, W>(acc, ring + slot * G::kStageBytes, lane, valid, L);
      ++n_done;
      __syncwarp();
      if (lane == 0 && pu < u1) issue_next();
    }
    if (aborted) break;
    if (RAW) {  // the no-fit record holds sum |x - y|^2 in its first word
      acc[0] += acc[1] + acc[2];
      acc[1] = acc[2] = 0.0;
    }
    const int64_t f = g * 32 + lane;
    if (f < F) {
      double2* rec = reinterpret_cast<double2*>(L.partial + ((size_t)f * n_tiles + t) * kStatDoubles);
#pragma unroll
      for (int e = 0; e < 7; ++e) rec[e] = make_double2(acc[2 * e], acc[2 * e + 1]);
      rec[7] = make_double2(acc[14], 0.0);
    }
  }

  // after an abort, copies this warp issued may still be landing (a withheld
  // stage has none)
  if (aborted && lane == 0) {
    for (int64_t j = n_done; j < n_issued; ++j)
      if (!(withheld && j == 0)) mbar_drain(&full[j % kLaneStages], (uint32_t)((j / kLaneStages) & 1), L.status);
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
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

int64_t lane_units(const FrameLaunch& L, int64_t tile) {
  return ((L.n_frames + 31) / 32) * ((L.lane_atoms + tile - 1) / tile);
}

template <int STRIDE, bool RAW, bool QUAD = false>
int lanes_occupancy() {
  using G = typename PickGeo<QUAD, STRIDE>::type;
  auto kern = rmsd_lanes_kernel<STRIDE, RAW, false, QUAD>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmemBytes);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kLaneWarps * 32, G::kSmemBytes) != cudaSuccess) b = 1;
  return std::max(b, 1);
}

// QUAD: L.n_frames is a multiple of 4 and the rows of the tensor map are
// quad rows of 4 frames (packed xyz, dense selection).
template <int STRIDE, bool RAW, bool W, bool QUAD = false>
cudaError_t launch_lanes(const FrameLaunch& L, cudaStream_t s) {
  using G = typename PickGeo<QUAD, STRIDE>::type;
  EncodeTiled enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap map;
  CUresult r;
  if (QUAD) {
    const cuuint64_t dims[2] = {(cuuint64_t)(L.n_atoms * 12), (cuuint64_t)(L.n_frames / 4)};
    const cuuint64_t strides[1] = {(cuuint64_t)(L.n_atoms * 48)};
    const cuuint32_t box[2] = {100, 8};
    const cuuint32_t estr[2] = {1, 1};
    r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(L.coords), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const cuuint64_t dims[2] = {(cuuint64_t)(L.lane_atoms * STRIDE), (cuuint64_t)L.n_frames};
    const cuuint64_t strides[1] = {(cuuint64_t)(L.n_atoms * STRIDE * 4)};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    float* base = const_cast<float*>(L.coords) + L.lane_atom0 * STRIDE;
    r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  auto kern = rmsd_lanes_kernel<STRIDE, RAW, W, QUAD>;
  static bool attr_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  kern<<<L.grid, kLaneWarps * 32, G::kSmemBytes, s>>>(map, L);
  return cudaGetLastError();
}

// Packed xyz frames whose stride is not a multiple of 16 bytes, streamed as
// quad rows: a dense selection only (the tensor map covers whole frames).
bool lanes_quad(const FrameLaunch& L) {
  return L.stride == 3 && (L.n_atoms & 3) != 0 && L.sel == nullptr && L.lane_atom0 == 0 &&
         L.lane_atoms == L.ref.n_sel && L.lane_y == L.ref.yc && L.lane_w == L.ref.w;
}

// y_exp[(sel[i] - a0)][c] = yc[i][c], w_exp[sel[i] - a0] = w ? w[i] : 1 (the
// buffers were zeroed; selection indices are strictly increasing)
__global__ void lanes_expand_kernel(const uint32_t* __restrict__ sel, int64_t n_sel, int64_t a0,
                                    const double* __restrict__ yc, const float* __restrict__ w,
                                    double* __restrict__ y_exp, float* __restrict__ w_exp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_sel; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = (int64_t)sel[i] - a0;
    y_exp[k * 3 + 0] = yc[i * 3 + 0];
    y_exp[k * 3 + 1] = yc[i * 3 + 1];
    y_exp[k * 3 + 2] = yc[i * 3 + 2];
    w_exp[k] = w ? w[i] : 1.0f;
  }
}

}  // namespace

cudaError_t launch_lanes_expand(const uint32_t* sel, int64_t n_sel, int64_t a0, const double* yc, const float* w,
                                double* y_exp, float* w_exp, cudaStream_t s) {
  if (n_sel <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<int64_t>((n_sel + 255) / 256, 4096);
  lanes_expand_kernel<<<grid, 256, 0, s>>>(sel, n_sel, a0, yc, w, y_exp, w_exp);
  return cudaGetLastError();
}

bool lanes_eligible(const FrameLaunch& L) {
  static int mode = -1;
  if (mode < 0) {
    // WMD_FRAMES_KERNEL=atoms: always the atom-major kernel; =noquad: not for
    // packed frames whose stride is not a multiple of 16 bytes
    const char* e = std::getenv("WMD_FRAMES_KERNEL");
    mode = (e && std::strcmp(e, "atoms") == 0) ? 0 : (e && std::strcmp(e, "noquad") == 0) ? 2 : 1;
  }
  if (!mode || L.lane_atoms <= 0 || L.n_frames <= 0) return false;
  if ((reinterpret_cast<uintptr_t>(L.coords + L.lane_atom0 * L.stride) & 15u) != 0) return false;
  if (L.stride != 4 && (L.n_atoms & 3) != 0) {
    // quad rows of 4 frames: whole frames of a dense selection, and enough
    // frames that the gathered tail (n_frames mod 4) stays small
    if (mode == 2 || !lanes_quad(L) || L.n_frames < 32) return false;
    return L.n_atoms * 12 < (int64_t(1) << 31) && L.n_frames < (int64_t(1) << 31);
  }
  if ((L.lane_atom0 + L.lane_atoms) * L.stride >= (int64_t(1) << 31) || L.n_frames >= (int64_t(1) << 31))
    return false;
  return true;
}

static int lanes_slots(const FrameLaunch& L, int sm_count) {
  static int occ[3] = {0, 0, 0};
  const int which = L.stride == 4 ? 1 : lanes_quad(L) ? 2 : 0;
  int& o = occ[which];
  if (o == 0) o = which == 1 ? lanes_occupancy<4, false>() : which == 2 ? lanes_occupancy<3, false, true>()
                                                                        : lanes_occupancy<3, false>();
  return sm_count * o * kLaneWarps;
}

// Active warps for `slots` warp slots: every warp gets the same number of
// whole units (the last one possibly fewer).
static int64_t lane_warps(const FrameLaunch& L, int64_t slots) {
  const int64_t units = lane_units(L, L.tile_atoms);
  const int64_t per = (units + slots - 1) / slots;
  return std::max<int64_t>(1, (units + per - 1) / per);
}

bool lanes_worthwhile(const FrameLaunch& L, int sm_count) {
  // fewer (256-atom tile, 32-frame group) units than two per SM: the
  // atom-major kernel's (tile, frame) items spread better
  return lane_units(L, 256) >= 2 * (int64_t)sm_count;
}

int lanes_tile(const FrameLaunch& L, int sm_count) {
  // Tile size from 2,048 down to 256 atoms minimising the busiest warp's
  // bytes: (units per warp) x (tile bytes + its 128-byte partial, written
  // and read back).  Large tiles mean few records; small ones balance short
  // runs (few frames or few atoms) over all warp slots.
  const int64_t slots = lanes_slots(L, sm_count);
  int64_t best = kLaneTile, best_cost = -1;
  for (int64_t tile = kLaneTile; tile >= 256; tile /= 2) {
    const int64_t per = (lane_units(L, tile) + slots - 1) / slots;
    const int64_t cost = per * (tile * L.stride * 4 + 256);
    if (best_cost < 0 || cost < best_cost) {
      best = tile;
      best_cost = cost;
    }
  }
  return (int)best;
}

int lanes_grid(const FrameLaunch& L, int sm_count) {
  return (int)((lane_warps(L, lanes_slots(L, sm_count)) + kLaneWarps - 1) / kLaneWarps);
}

cudaError_t launch_lanes_forward(const FrameLaunch& L, bool raw, cudaStream_t s) {
  FrameLaunch K = L;
  const bool w = L.lane_w != nullptr;
  if (lanes_quad(L)) {
    // whole quad rows here; the last n_frames mod 4 frames by the gathered
    // kernel into the same partial layout
    const int64_t main = L.n_frames & ~int64_t(3);
    if (main > 0) {  // a batch of fewer than 4 frames has no quad row
      K.n_frames = main;
      K.lane_warps = (int)lane_warps(K, (int64_t)L.grid * kLaneWarps);
      cudaError_t e = w ? (raw ? launch_lanes<3, true, true, true>(K, s) : launch_lanes<3, false, true, true>(K, s))
                        : (raw ? launch_lanes<3, true, false, true>(K, s) : launch_lanes<3, false, false, true>(K, s));
      if (e != cudaSuccess || main == L.n_frames) return e;
    }
    FrameLaunch T = L;
    T.coords = L.coords + (size_t)main * L.n_atoms * 3;
    T.n_frames = L.n_frames - main;
    T.partial = L.partial + (size_t)main * frame_tiles(L) * kStatDoubles;
    static int sms[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!sms[dev]) cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
    return launch_gather_partials(T, raw, sms[dev], s);
  }
  K.lane_warps = (int)lane_warps(L, (int64_t)L.grid * kLaneWarps);
  if (L.stride == 4) {
    if (w) return raw ? launch_lanes<4, true, true>(K, s) : launch_lanes<4, false, true>(K, s);
    return raw ? launch_lanes<4, true, false>(K, s) : launch_lanes<4, false, false>(K, s);
  }
  if (w) return raw ? launch_lanes<3, true, true>(K, s) : launch_lanes<3, false, true>(K, s);
  return raw ? launch_lanes<3, true, false>(K, s) : launch_lanes<3, false, false>(K, s);
}

}  // namespace wmd

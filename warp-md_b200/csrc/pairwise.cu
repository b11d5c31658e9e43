// pairwise.cu -- all-pairs frame x frame RMSD matrix.
//
// Reference behaviour: PairwiseRmsdPlan::finalize
// (crates/traj-engine/src/plans/rmsd/plan.rs:593-674) -- CPU only, FP64, one
// Kabsch SVD per pair (rmsd_aligned, plan.rs:1112-1159) or a raw RMSD
// (rmsd_raw, plan.rs:1081-1091); symmetric fill, zero diagonal, all zeros when
// fewer than two atoms are selected.
//
// Here every frame is centred once (FP64 centroid, coordinates stored in the
// mode's precision, G_i = sum |x_i - c_i|^2 of the stored values in FP64), the
// nine covariance entries of all pairs are the 3N x 3N Gram matrix of the
// centred frames, and a per-pair FP64 epilogue turns each 3x3 block into an
// RMSD (QCP for "rms"; G_i + G_j - 2 tr H + n |c_i - c_j|^2 for "nofit").
//
// This file holds the SIMT forms (FP32 and FP64 accumulation, the plain GPU
// baseline and the on-GPU accuracy reference); the tensor-core forms live in
// pairwise_tc.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/warpmd_rmsd.h"
#include "pairwise.h"
#include "pairwise_tc.h"
#include "device_util.cuh"
#include "qcp.cuh"

namespace wmd {

constexpr int kPairKc = 32;      // atoms per K step of the SIMT tiles
constexpr int kPanelFrames = 32;  // frames per panel (= per SIMT block side)
constexpr int kPanelRows = 3 * kPanelFrames;

// Centres each selected frame (one CTA per frame) and stores it in the panel
// layout the SIMT tiles read: panel b = frames [32b, 32b + 32) as
// P[b][k][3 (f - 32b) + c] (k = atom, zero padded to n_pad), so one K step of
// a tile is one contiguous 32 x 96 block.  G_f is the FP64 sum of squares of
// the stored (rounded) values, so H and G describe the same coordinates.
template <typename T>
__global__ void __launch_bounds__(256) pair_prep(const float* __restrict__ coords, int64_t n_atoms, int stride,
                                                 const uint32_t* __restrict__ sel, int64_t n_sel, int64_t n_pad,
                                                 T* __restrict__ xc, double* __restrict__ gsum,
                                                 double* __restrict__ cen, int* status) {
  __shared__ double red[8][4];
  const int64_t f = blockIdx.x;
  const float* fr = coords + (size_t)f * n_atoms * stride;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
    int64_t idx = sel ? (int64_t)sel[k] : k;
    if (idx >= n_atoms) {  // bad device-side selection: report, read atom 0
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
  const double inv = n_sel > 0 ? 1.0 / (double)n_sel : 0.0;
  c[0] *= inv; c[1] *= inv; c[2] *= inv;
  __syncthreads();
  T* panel = xc + (size_t)(f / kPanelFrames) * n_pad * kPanelRows + 3 * (f % kPanelFrames);
  double g = 0;
  for (int64_t k = threadIdx.x; k < n_pad; k += blockDim.x) {
    T* dst = panel + (size_t)k * kPanelRows;
    if (k < n_sel) {
      int64_t idx = sel ? (int64_t)sel[k] : k;
      if (idx >= n_atoms) idx = 0;
      const float* p = fr + idx * stride;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const T v = (T)((double)p[q] - c[q]);
        dst[q] = v;
        g += (double)v * (double)v;
      }
    } else {
      dst[0] = T(0); dst[1] = T(0); dst[2] = T(0);
    }
  }
  for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
  if (lane == 0) red[warp][3] = g;
  __syncthreads();
  if (threadIdx.x == 0) {
    double gt = 0;
    for (int w = 0; w < 8; ++w) gt += red[w][3];
    gsum[f] = gt;
    cen[f * 3 + 0] = c[0]; cen[f * 3 + 1] = c[1]; cen[f * 3 + 2] = c[2];
  }
}

// Per-pair epilogue shared by every pairwise form: h = covariance block of
// frames (i, j), returns the RMSD.
__device__ __forceinline__ double pair_rmsd(const double h[9], double gi, double gj, const double* ci,
                                            const double* cj, double n, int metric) {
  if (metric == WMD_PAIR_NOFIT) {
    const double d0 = ci[0] - cj[0], d1 = ci[1] - cj[1], d2 = ci[2] - cj[2];
    const double s = gi + gj - 2.0 * (h[0] + h[4] + h[8]) + n * (d0 * d0 + d1 * d1 + d2 * d2);
    return s > 0.0 ? sqrt(s / n) : 0.0;
  }
  const QcpOut q = qcp_lambda(h, 0.5 * (gi + gj));
  return sqrt(msd_from(gi, gj, q.lambda, n));
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Two consecutive T values from shared memory (8 or 16 bytes, aligned).
template <typename T>
struct Pair2 { T x, y; };

// SIMT tile over one (row panel, column panel) pair of 32 frames each: 16 x 16
// threads, thread (ty, tx) owns frames 2ty, 2ty+1 x 2tx, 2tx+1 -- four full 3x3
// covariance blocks, 36 FMAs per atom against 6 vector shared loads.  K steps
// of 32 atoms are double-buffered with cp.async.  Only pairs i < j are
// finished (FP64 epilogue) and written to both (i, j) and (j, i).
template <typename T>
__global__ void __launch_bounds__(256) pair_tile_simt(const T* __restrict__ xc, const double* __restrict__ gsum,
                                                      const double* __restrict__ cen, int64_t F, int64_t n_pad,
                                                      double n, int metric, float* __restrict__ out, int part,
                                                      int parts) {
  constexpr int kStep = kPairKc * kPanelRows;  // elements per panel K step
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);      // [2][kPairKc][96]
  T* Bs = As + 2 * kStep;
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bi > bj || bi % parts != part) return;
  const int64_t I0 = (int64_t)bi * kPanelFrames, J0 = (int64_t)bj * kPanelFrames;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const T* pa = xc + (size_t)bi * n_pad * kPanelRows;
  const T* pb = xc + (size_t)bj * n_pad * kPanelRows;
  constexpr int kVec = 16 / sizeof(T);         // elements per 16-byte copy
  constexpr int kCopies = kStep / kVec;        // per operand per step
  auto load = [&](int buf, int64_t k0) {
    const T* ga = pa + (size_t)k0 * kPanelRows;
    const T* gb = pb + (size_t)k0 * kPanelRows;
    for (int c = tid; c < kCopies; c += 256) {
      cp_async16(As + buf * kStep + c * kVec, ga + c * kVec);
      cp_async16(Bs + buf * kStep + c * kVec, gb + c * kVec);
    }
    cp_async_commit();
  };
  T acc[2][2][9];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 9; ++e) acc[a][b][e] = T(0);
  const int steps = (int)(n_pad / kPairKc);
  load(0, 0);
  for (int st = 0; st < steps; ++st) {
    const int buf = st & 1;
    if (st + 1 < steps) {
      load(buf ^ 1, (int64_t)(st + 1) * kPairKc);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const T* A = As + buf * kStep + 6 * ty;
    const T* B = Bs + buf * kStep + 6 * tx;
#pragma unroll 4
    for (int kk = 0; kk < kPairKc; ++kk) {
      T xa[6], xb[6];
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        const Pair2<T> qa = *reinterpret_cast<const Pair2<T>*>(A + kk * kPanelRows + 2 * v);
        const Pair2<T> qb = *reinterpret_cast<const Pair2<T>*>(B + kk * kPanelRows + 2 * v);
        xa[2 * v] = qa.x; xa[2 * v + 1] = qa.y;
        xb[2 * v] = qb.x; xb[2 * v + 1] = qb.y;
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int q = 0; q < 3; ++q)
              acc[a][b][p * 3 + q] = fma(xa[3 * a + p], xb[3 * b + q], acc[a][b][p * 3 + q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int64_t i = I0 + 2 * ty + a;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int64_t j = J0 + 2 * tx + b;
      if (i < j && j < F) {
        double h[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) h[e] = (double)acc[a][b][e];
        const float v = (float)pair_rmsd(h, gsum[i], gsum[j], cen + i * 3, cen + j * 3, n, metric);
        out[(size_t)i * F + j] = v;
        out[(size_t)j * F + i] = v;
      }
    }
  }
}

void pairwise_workspace_free(PairwiseWorkspace& w) {
  if (w.centred) cudaFree(w.centred);
  if (w.gsum) cudaFree(w.gsum);
  if (w.cen) cudaFree(w.cen);
  if (w.extra) cudaFree(w.extra);
  w = PairwiseWorkspace();
}

static int grow(void** p, size_t* have, size_t want, std::string* msg) {
  if (*p && *have >= want) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(p, std::max<size_t>(want, 256));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    *msg = std::string("cuda driver error: pairwise workspace allocation failed: ") + cudaGetErrorString(e);
    return WMD_ERR_OOM;
  }
  *have = std::max<size_t>(want, 256);
  return 0;
}

template <typename T>
static cudaError_t run_simt(PairwiseWorkspace& w, int64_t F, int64_t n_pad, int64_t n_sel, int metric, float* out,
                            cudaStream_t s) {
  const size_t smem = (size_t)4 * kPairKc * kPanelRows * sizeof(T);
  auto kern = pair_tile_simt<T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const unsigned nb = (unsigned)((F + kPanelFrames - 1) / kPanelFrames);
  dim3 grid(nb, nb);
  kern<<<grid, 256, smem, s>>>(static_cast<const T*>(w.centred), w.gsum, w.cen, F, n_pad, (double)n_sel, metric, out,
                               w.part, w.parts);
  return cudaGetLastError();
}

int pairwise_run(PairwiseWorkspace& w, int sm_count, const float* coords, int64_t n_frames, int64_t n_atoms,
                 int stride, const uint32_t* sel, int64_t n_sel, int metric, int mode, float* out, int* status,
                 cudaStream_t s, std::string* msg) {
  const size_t out_bytes = (size_t)n_frames * n_frames * sizeof(float);
  cudaError_t e = cudaMemsetAsync(out, 0, out_bytes, s);
  if (e != cudaSuccess) {
    *msg = std::string("cuda driver error: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  if (n_sel < 2 || n_frames < 2) return 0;  // all zeros (plan.rs:604-610)

  if (mode == WMD_MODE_I8X3 || mode == WMD_MODE_I8X2)
    return pairwise_tc_run(w, sm_count, coords, n_frames, n_atoms, stride, sel, n_sel, metric,
                           mode == WMD_MODE_I8X3 ? 3 : 2, out, status, w.wait, s, msg);

  const bool f64 = mode == WMD_MODE_FP64;
  const int64_t n_pad = (n_sel + kPairKc - 1) / kPairKc * kPairKc;
  const size_t elem = f64 ? sizeof(double) : sizeof(float);
  const int64_t panels = (n_frames + kPanelFrames - 1) / kPanelFrames;
  int rc = grow(&w.centred, &w.centred_bytes, (size_t)panels * n_pad * kPanelRows * elem, msg);
  if (rc) return rc;
  // frames past the end of the last panel stay zero
  e = cudaMemsetAsync(w.centred, 0, (size_t)panels * n_pad * kPanelRows * elem, s);
  if (e != cudaSuccess) {
    *msg = std::string("cuda driver error: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  if (w.frames_cap < (size_t)n_frames) {
    if (w.gsum) cudaFree(w.gsum);
    if (w.cen) cudaFree(w.cen);
    w.gsum = nullptr;
    w.cen = nullptr;
    w.frames_cap = 0;
    if ((e = cudaMalloc(&w.gsum, n_frames * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&w.cen, n_frames * 3 * sizeof(double))) != cudaSuccess) {
      cudaGetLastError();
      *msg = std::string("cuda driver error: pairwise workspace allocation failed: ") + cudaGetErrorString(e);
      return WMD_ERR_OOM;
    }
    w.frames_cap = n_frames;
  }
  if (f64)
    pair_prep<double><<<(unsigned)n_frames, 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, n_pad,
                                                         static_cast<double*>(w.centred), w.gsum, w.cen, status);
  else
    pair_prep<float><<<(unsigned)n_frames, 256, 0, s>>>(coords, n_atoms, stride, sel, n_sel, n_pad,
                                                        static_cast<float*>(w.centred), w.gsum, w.cen, status);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = f64 ? run_simt<double>(w, n_frames, n_pad, n_sel, metric, out, s)
                                : run_simt<float>(w, n_frames, n_pad, n_sel, metric, out, s);
  if (e != cudaSuccess) {
    *msg = std::string("cuda driver error: pairwise launch: ") + cudaGetErrorString(e);
    return WMD_ERR_CUDA;
  }
  return 0;
}

}  // namespace wmd

// cluster.cu -- DBSCAN over the all-pairs RMSD matrix (TrajectoryClusterPlan,
// method "dbscan": crates/traj-engine/src/plans/analysis/clustering.rs:160-190,
// 269-383).
//
// The reference runs the textbook sequential DBSCAN over the triangular f32
// matrix.  Its result is a function of the matrix alone, which this file
// computes in parallel:
//   * a point is core when at least min_samples points (itself included) lie
//     within eps;
//   * clusters are the connected components of core points under d <= eps,
//     numbered in increasing order of their smallest core index (the order in
//     which the sequential outer loop starts them);
//   * a non-core point takes the smallest cluster id among its core neighbours
//     (the first cluster whose expansion reaches it), or -1 (noise);
//   * a cluster's centroid is the member with the smallest FP64 sum of
//     distances to all members, summed in index order, ties to the lowest
//     index (clustering.rs:347-373).
// Kernels: row degrees; union-find over core-core edges (lock-free, larger
// root hooked under the smaller, so each root is its component's minimum);
// root ranking; labels; sizes; medoid sums and the two-pass argmin.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "cluster.h"
#include "device_util.cuh"

namespace wmd {
namespace {

constexpr int kRowThreads = 256;

__device__ __forceinline__ bool within(float d, double eps) { return (double)d <= eps; }

// deg[i] = #{j : d(i, j) <= eps}, the diagonal counted as 0.
__global__ void __launch_bounds__(kRowThreads) degree_kernel(const float* __restrict__ D, int64_t n, double eps,
                                                             int64_t min_samples, uint8_t* __restrict__ core) {
  __shared__ int red[kRowThreads / 32];
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const float* row = D + (size_t)i * n;
    int c = 0;
    for (int64_t j = threadIdx.x; j < n; j += kRowThreads) c += (j == i || within(row[j], eps)) ? 1 : 0;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kRowThreads / 32; ++w) t += red[w];
      core[i] = (int64_t)t >= min_samples ? 1 : 0;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int find_root(const int* parent, int x) {
  // parents only ever point to smaller indices, so this takes at most x steps
  // (loads bypass L1, so links made by other SMs are seen)
  int p = __ldcg(parent + x);
  while (p != x) {
    x = p;
    p = __ldcg(parent + x);
  }
  return x;
}

// Scratch layout (dbscan_scratch_bytes): parent, root, cluster_of_root as int
// [n] each, sum as double [n], core as byte [n].
struct DbLayout {
  int* parent;
  int* root;
  int* cluster_of_root;
  double* sum;
  uint8_t* core;
  __host__ __device__ DbLayout(void* scratch, int64_t n) {
    char* p = static_cast<char*>(scratch);
    parent = reinterpret_cast<int*>(p);
    root = parent + n;
    cluster_of_root = root + n;
    sum = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(cluster_of_root + n) + 7) & ~uintptr_t(7));
    core = reinterpret_cast<uint8_t*>(sum + n);
  }
};

__global__ void init_parent_kernel(int* parent, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parent[i] = (int)i;
}

// Union of every core-core pair within eps, i < j: a block per row i.
__global__ void __launch_bounds__(kRowThreads) union_kernel(const float* __restrict__ D, int64_t n, double eps,
                                                            const uint8_t* __restrict__ core, int* parent,
                                                            int* status) {
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    if (!core[i]) continue;
    const float* row = D + (size_t)i * n;
    for (int64_t j = i + 1 + threadIdx.x; j < n; j += kRowThreads) {
      if (!core[j] || !within(row[j], eps)) continue;
      int a = (int)i, b = (int)j;
      // lock-free union: hook the larger root under the smaller; a failed CAS
      // means another thread linked that root (at most n - 1 links happen in
      // all), so look again -- with a cap that reports instead of spinning on
      int tries = 0;
      for (;; ++tries) {
        if (tries > (1 << 24)) {
          atomicOr(status, kClusterStatusRetries);
          break;
        }
        a = find_root(parent, a);
        b = find_root(parent, b);
        if (a == b) break;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) break;
        a = lo;
        b = old;
      }
    }
  }
}

// root[i] = component root of core point i (-1 for non-core); is_root flags.
__global__ void roots_kernel(const int* parent, const uint8_t* core, int64_t n, int* root) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) root[i] = core[i] ? find_root(parent, (int)i) : -1;
}

// cluster_of_root[i] = rank of root i among all roots (one block, in order).
__global__ void __launch_bounds__(1024) rank_roots_kernel(const int* root, int64_t n, int* cluster_of_root,
                                                          int* n_clusters) {
  __shared__ int carry;
  __shared__ int warp_sums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const int flag = (i < n && root[i] == (int)i) ? 1 : 0;
    // block-wide exclusive scan of flag
    int v = flag;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
      int w = warp_sums[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += u;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const int incl = v + (warp > 0 ? warp_sums[warp - 1] : 0);
    if (i < n) cluster_of_root[i] = flag ? carry + incl - 1 : -1;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_clusters = carry;
}

// Labels: core -> its component's cluster; non-core -> the smallest cluster of
// a core neighbour within eps, or -1.  A block per point.
__global__ void __launch_bounds__(kRowThreads) label_kernel(const float* __restrict__ D, int64_t n, double eps,
                                                            const uint8_t* __restrict__ core,
                                                            const int* __restrict__ root,
                                                            const int* __restrict__ cluster_of_root,
                                                            int* __restrict__ labels) {
  __shared__ int red[kRowThreads / 32];
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    if (core[i]) {
      if (threadIdx.x == 0) labels[i] = cluster_of_root[root[i]];
      continue;
    }
    const float* row = D + (size_t)i * n;
    int best = 0x7fffffff;
    for (int64_t j = threadIdx.x; j < n; j += kRowThreads)
      if (j != i && core[j] && within(row[j], eps)) best = min(best, cluster_of_root[root[j]]);
    for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
      int b = 0x7fffffff;
      for (int w = 0; w < kRowThreads / 32; ++w) b = min(b, red[w]);
      labels[i] = b == 0x7fffffff ? -1 : b;
    }
    __syncthreads();
  }
}

__global__ void sizes_kernel(const int* labels, int64_t n, unsigned* sizes) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && labels[i] >= 0) atomicAdd(sizes + labels[i], 1u);
}

// sum[i] = sum over members j of i's cluster, in index order, of d(i, j), FP64
// (the reference's sequential loop).  A warp per point reads its row
// coalesced.  The lanes' strided partial sums equal the sequential sum
// whenever no addition in either order rounds: every term is a multiple of
// 2^low (low = the smallest term's last mantissa bit) and the total is below
// 2^(53 + low), so every partial sum of any subset is representable.  Rows
// that miss that bound (tiny distances next to large ones) take the
// sequential loop on lane 0.
__global__ void __launch_bounds__(256) medoid_sum_kernel(const float* __restrict__ D, int64_t n,
                                                         const int* __restrict__ labels, double* __restrict__ sum,
                                                         unsigned long long* __restrict__ best_bits) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int c = labels[i];
    if (c < 0) continue;  // warp-uniform
    const float* row = D + (size_t)i * n;
    double s = 0.0;
    int low = 1 << 20;  // lowest set-able mantissa bit over the lane's terms
    for (int64_t j = lane; j < n; j += 32) {
      if (j == i || __ldg(labels + j) != c) continue;
      const float v = __ldg(row + j);
      if (v == 0.0f) continue;
      const int e = (int)((__float_as_uint(v) >> 23) & 0xffu);
      low = min(low, (e == 0 ? 1 : e) - 150);  // value = m * 2^(e - 150), subnormals 2^-149
      s += (double)v;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      low = min(low, __shfl_xor_sync(0xffffffffu, low, o));
    }
    // the same total on every lane; s >= the exact sum's lower neighbour
    const bool exact = low == (1 << 20) || s < ldexp(1.0, 53 + low) * 0.5;
    if (lane == 0) {
      if (!exact) {
        s = 0.0;
        for (int64_t j = 0; j < n; ++j)
          if (labels[j] == c) s += j == i ? 0.0 : (double)row[j];
      }
      sum[i] = s;
      // non-negative doubles order like their bit patterns
      atomicMin(best_bits + c, (unsigned long long)__double_as_longlong(s));
    }
  }
}

__global__ void medoid_pick_kernel(int64_t n, const int* labels, const double* sum,
                                   const unsigned long long* best_bits, unsigned* centroid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = labels[i];
  if (c < 0) return;
  if ((unsigned long long)__double_as_longlong(sum[i]) == best_bits[c]) atomicMin(centroid + c, (unsigned)i);
}

// ---------------------------------------------------------------------------
// k-means (TrajectoryClusterPlan, method "kmeans": clustering.rs:191-205,
// 376-548).  Features are the selection's coordinates after superposition
// onto frame 0, in FP64; every distance and every sum runs in the reference's
// order (features in order, samples in index order), so assignments are the
// reference's up to exact FP64 ties.
// ---------------------------------------------------------------------------


// feat[i][3a + c] = (R_i x_ia + t_i)_c
template <int STRIDE>
__global__ void kmeans_features_kernel(const float* __restrict__ coords, int64_t n_frames, int64_t n_atoms,
                                       const uint32_t* __restrict__ sel, int64_t n_sel,
                                       const double* __restrict__ xf, double* __restrict__ feat) {
  const int64_t total = n_frames * n_sel;
  for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < total; it += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = it / n_sel, a = it - f * n_sel;
    const int64_t atom = sel ? (int64_t)sel[a] : a;
    const float* p = coords + ((size_t)f * n_atoms + atom) * STRIDE;
    const double* x = xf + f * 16;
    const double p0 = p[0], p1 = p[1], p2 = p[2];
    double* o = feat + (size_t)f * n_sel * 3 + a * 3;
    o[0] = x[0] * p0 + x[1] * p1 + x[2] * p2 + x[9];
    o[1] = x[3] * p0 + x[4] * p1 + x[5] * p2 + x[10];
    o[2] = x[6] * p0 + x[7] * p1 + x[8] * p2 + x[11];
  }
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Assignment tiles: kAsRows samples x (8 or 16) centers per block, features
// staged through shared memory kAsTile at a time (coalesced row loads).  A
// warp owns CPT (1 for k <= 8, else 2) centers for its 32 samples (lane =
// sample); every distance is the sequential sum over features in order with
// an unfused multiply then add, as the reference's sq_dist.  Zero padding past
// nf adds exact zeros.  The next tile is loaded into registers while the
// current one is used (two shared buffers, one barrier per tile).
constexpr int kAsRows = 32;
constexpr int kAsWarps = 8;
constexpr int kAsTile = 48;
constexpr int kAsPerThread = kAsRows * kAsTile / (kAsWarps * 32);  // x values per thread and tile

// labels[i] = argmin_c |feat[i] - centers[c]|^2 (first minimum), or, when
// own_labels is given, dist[i] = the distance to centers[own_labels[i]] and
// the per-cluster minimum as ordered bits in best_bits.
template <int CPT>
__global__ void __launch_bounds__(kAsWarps * 32) kmeans_assign_kernel(
    const double* __restrict__ feat, int64_t n, int64_t nf, const double* __restrict__ centers, int k,
    int* __restrict__ labels, const int* __restrict__ own_labels, double* __restrict__ dist,
    unsigned long long* __restrict__ best_bits) {
  constexpr int kAsCenters = kAsWarps * CPT;
  constexpr int kAsCPerThread = kAsCenters * kAsTile / (kAsWarps * 32);  // center values per thread and tile
  __shared__ double xs[2][kAsRows][kAsTile + 1];
  __shared__ double cs[2][kAsCenters][kAsTile];
  __shared__ double dsm[kAsCenters][kAsRows];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t row0 = (int64_t)blockIdx.x * kAsRows;
  const int64_t my_row = row0 + lane;
  const int own = (own_labels && warp == 0 && my_row < n) ? own_labels[my_row] : -1;
  double best_d = __longlong_as_double(0x7ff0000000000000ll);  // +inf
  double own_d = 0.0;
  int best = 0;
  const int64_t n_tiles = (nf + kAsTile - 1) / kAsTile;
  for (int c0 = 0; c0 < k; c0 += kAsCenters) {
    double d[CPT];
#pragma unroll
    for (int p = 0; p < CPT; ++p) d[p] = 0.0;
    double xr[kAsPerThread], cr[kAsCPerThread];
    auto fetch = [&](int64_t j0) {  // tile j0 into registers (zero past nf / n / k)
#pragma unroll
      for (int m = 0; m < kAsPerThread; ++m) {
        const int e = tid + m * kAsWarps * 32;
        const int r = e / kAsTile, q = e - r * kAsTile;
        const int64_t row = row0 + r;
        xr[m] = (row < n && j0 + q < nf) ? __ldg(feat + (size_t)row * nf + j0 + q) : 0.0;
      }
#pragma unroll
      for (int m = 0; m < kAsCPerThread; ++m) {
        const int e = tid + m * kAsWarps * 32;
        const int cc = e / kAsTile, q = e - cc * kAsTile;
        const int c = c0 + cc;
        cr[m] = (c < k && j0 + q < nf) ? __ldg(centers + (size_t)c * nf + j0 + q) : 0.0;
      }
    };
    auto stash = [&](int buf) {
#pragma unroll
      for (int m = 0; m < kAsPerThread; ++m) {
        const int e = tid + m * kAsWarps * 32;
        const int r = e / kAsTile, q = e - r * kAsTile;
        xs[buf][r][q] = xr[m];
      }
#pragma unroll
      for (int m = 0; m < kAsCPerThread; ++m) {
        const int e = tid + m * kAsWarps * 32;
        const int cc = e / kAsTile, q = e - cc * kAsTile;
        cs[buf][cc][q] = cr[m];
      }
    };
    fetch(0);
    stash(0);
    __syncthreads();
    for (int64_t tt = 0; tt < n_tiles; ++tt) {
      const int buf = (int)(tt & 1);
      if (tt + 1 < n_tiles) fetch((tt + 1) * kAsTile);
#pragma unroll 8
      for (int q = 0; q < kAsTile; ++q) {
        const double x = xs[buf][lane][q];
#pragma unroll
        for (int p = 0; p < CPT; ++p) {
          const double e = x - cs[buf][warp * CPT + p][q];
          d[p] = __dadd_rn(d[p], __dmul_rn(e, e));
        }
      }
      // the other buffer was last read before the previous barrier
      if (tt + 1 < n_tiles) stash(buf ^ 1);
      __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < CPT; ++p) dsm[warp * CPT + p][lane] = d[p];
    __syncthreads();
    if (warp == 0) {
      for (int cc = 0; cc < kAsCenters && c0 + cc < k; ++cc) {
        const double v = dsm[cc][lane];
        if (v < best_d) {
          best_d = v;
          best = c0 + cc;
        }
        if (c0 + cc == own) own_d = v;
      }
    }
    __syncthreads();
  }
  if (warp != 0 || my_row >= n) return;
  if (!own_labels) {
    labels[my_row] = best;
  } else {
    dist[my_row] = own_d;
    if (own >= 0) atomicMin(best_bits + own, (unsigned long long)__double_as_longlong(own_d));
  }
}

// Per-cluster sums in sample order.  Block = (128 feature columns, one
// cluster); each warp scans the labels 32 at a time and queues its members'
// indices in index order (ballot + prefix count).  Every 32 queued rows each
// lane prefetches its column of them into shared memory with cp.async (8
// bytes per row, no registers held), and adds the previous batch from the
// other buffer meanwhile; each column's sum stays sequential in index order.
constexpr int kSumWarps = 4;
constexpr int kSumBatch = 32;
constexpr size_t kSumSmem = (size_t)kSumWarps * 2 * kSumBatch * 32 * sizeof(double);

__global__ void __launch_bounds__(kSumWarps * 32) kmeans_sums_kernel(const double* __restrict__ feat, int64_t n,
                                                                     int64_t nf, const int* __restrict__ labels,
                                                                     int k, double* __restrict__ sums,
                                                                     int* __restrict__ counts) {
  extern __shared__ double sum_smem[];
  __shared__ int queue[kSumWarps][2 * kSumBatch];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.y;
  const int64_t col0 = ((int64_t)blockIdx.x * kSumWarps + warp) * 32;
  if (col0 >= nf) return;  // warp-uniform
  const int64_t col = col0 + lane;
  const bool live = col < nf;
  int* q = queue[warp];
  double* buf = sum_smem + (size_t)warp * 2 * kSumBatch * 32;  // [2][kSumBatch][32]
  double acc = 0.0;
  int m = 0, cnt = 0, pending = -1, pending_take = 0, nb = 0;
  // rows q[0..take) into buffer b (this lane's column)
  auto issue = [&](int b, int take) {
    double* dst = buf + (size_t)b * kSumBatch * 32 + lane;
    if (live)
      for (int p = 0; p < take; ++p) cp_async8(dst + p * 32, feat + (size_t)q[p] * nf + col);
    cp_async_commit();
  };
  auto consume = [&](int b, int take) {
    const double* src = buf + (size_t)b * kSumBatch * 32 + lane;
    for (int p = 0; p < take; ++p) acc += src[p * 32];
  };
  // labels are read kSumAhead chunks at a time, so that the scan does not
  // wait for one load per 32 samples
  constexpr int kSumAhead = 8;
  for (int64_t i0 = 0; i0 < n; i0 += 32 * kSumAhead) {
    int lab[kSumAhead];
#pragma unroll
    for (int u = 0; u < kSumAhead; ++u) {
      const int64_t i = i0 + u * 32 + lane;
      lab[u] = i < n ? __ldg(labels + i) : -1;
    }
#pragma unroll
    for (int u = 0; u < kSumAhead; ++u) {
      const int64_t i = i0 + u * 32 + lane;
      const bool mine = lab[u] == c;
      const unsigned mask = __ballot_sync(0xffffffffu, mine);
      if (mine) q[m + __popc(mask & ((1u << lane) - 1u))] = (int)i;
      m += __popc(mask);
      cnt += __popc(mask);
      __syncwarp();
      if (m >= kSumBatch) {
        const int b = nb & 1;
        issue(b, kSumBatch);
        ++nb;
        if (pending >= 0) {
          cp_async_wait<1>();  // the previous batch has landed
          consume(pending, pending_take);
        }
        pending = b;
        pending_take = kSumBatch;
        const int rest = m - kSumBatch;  // < 32
        const int t = lane < rest ? q[kSumBatch + lane] : 0;
        __syncwarp();
        if (lane < rest) q[lane] = t;
        m = rest;
        __syncwarp();
      }
    }
  }
  if (m > 0) {
    const int b = nb & 1;
    issue(b, m);
    if (pending >= 0) {
      cp_async_wait<1>();
      consume(pending, pending_take);
    }
    pending = b;
    pending_take = m;
  }
  cp_async_wait<0>();
  if (pending >= 0) consume(pending, pending_take);
  if (live) sums[(size_t)c * nf + col] = acc;
  if (col == 0) counts[c] = cnt;
}

// New centers: sums / count, or the sample reseed[c] for an empty cluster;
// shift[c] = |old - new| with the squares added in feature order (thread 0
// over a shared-memory tile).  A block per cluster.
constexpr int kCtrTile = 2048;

__global__ void __launch_bounds__(256) kmeans_centers_kernel(const double* __restrict__ feat, int64_t nf,
                                                             const double* __restrict__ sums,
                                                             const int* __restrict__ counts,
                                                             const int64_t* __restrict__ reseed,
                                                             const double* __restrict__ old_c,
                                                             double* __restrict__ new_c, double* __restrict__ shift) {
  __shared__ double sq[kCtrTile];
  const int c = blockIdx.x;
  const int64_t src = reseed[c];
  const double inv = counts[c] > 0 ? 1.0 / (double)counts[c] : 0.0;
  double s = 0.0;
  for (int64_t j0 = 0; j0 < nf; j0 += kCtrTile) {
    const int tw = (int)min((int64_t)kCtrTile, nf - j0);
    for (int j = threadIdx.x; j < tw; j += blockDim.x) {
      const size_t at = (size_t)c * nf + j0 + j;
      const double v = src >= 0 ? feat[(size_t)src * nf + j0 + j] : sums[at] * inv;
      new_c[at] = v;
      const double e = old_c[at] - v;
      sq[j] = __dmul_rn(e, e);
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int j = 0; j < tw; ++j) s = __dadd_rn(s, sq[j]);
    __syncthreads();
  }
  if (threadIdx.x == 0) shift[c] = sqrt(s);
}

__global__ void kmeans_gather_kernel(const double* __restrict__ feat, int64_t nf, const int64_t* __restrict__ idx,
                                     double* __restrict__ centers) {
  const int c = blockIdx.x;
  for (int64_t j = threadIdx.x; j < nf; j += blockDim.x) centers[(size_t)c * nf + j] = feat[(size_t)idx[c] * nf + j];
}

}  // namespace

size_t dbscan_scratch_bytes(int64_t n) { return (size_t)n * (3 * sizeof(int) + sizeof(double) + 1) + 64; }

cudaError_t dbscan_run(const float* D, int64_t n, double eps, int64_t min_samples, void* scratch, int* labels,
                       int* n_clusters_dev, int* status, int sm_count, cudaStream_t s) {
  DbLayout L(scratch, n);
  const unsigned rows = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n, (int64_t)sm_count * 16));
  const unsigned lin = (unsigned)((n + 255) / 256);
  degree_kernel<<<rows, kRowThreads, 0, s>>>(D, n, eps, min_samples, L.core);
  init_parent_kernel<<<lin, 256, 0, s>>>(L.parent, n);
  union_kernel<<<rows, kRowThreads, 0, s>>>(D, n, eps, L.core, L.parent, status);
  roots_kernel<<<lin, 256, 0, s>>>(L.parent, L.core, n, L.root);
  rank_roots_kernel<<<1, 1024, 0, s>>>(L.root, n, L.cluster_of_root, n_clusters_dev);
  label_kernel<<<rows, kRowThreads, 0, s>>>(D, n, eps, L.core, L.root, L.cluster_of_root, labels);
  return cudaGetLastError();
}

cudaError_t dbscan_summary(const float* D, int64_t n, const int* labels, int64_t n_clusters, void* scratch,
                           unsigned* sizes, unsigned* centroids, unsigned long long* best_bits, cudaStream_t s) {
  DbLayout L(scratch, n);
  cudaError_t e;
  if (n_clusters == 0) return cudaSuccess;
  if ((e = cudaMemsetAsync(sizes, 0, (size_t)n_clusters * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(centroids, 0xff, (size_t)n_clusters * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(best_bits, 0xff, (size_t)n_clusters * sizeof(unsigned long long), s)) != cudaSuccess)
    return e;
  const unsigned lin = (unsigned)((n + 255) / 256);
  sizes_kernel<<<lin, 256, 0, s>>>(labels, n, sizes);
  const unsigned rows = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, 148 * 16));
  medoid_sum_kernel<<<rows, 256, 0, s>>>(D, n, labels, L.sum, best_bits);
  medoid_pick_kernel<<<lin, 256, 0, s>>>(n, labels, L.sum, best_bits, centroids);
  return cudaGetLastError();
}

}  // namespace wmd

namespace wmd {

cudaError_t kmeans_features(const float* coords, int64_t n_frames, int64_t n_atoms, int stride, const uint32_t* sel,
                            int64_t n_sel, const double* xf, double* feat, int sm_count, cudaStream_t s) {
  const int64_t total = n_frames * n_sel;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)sm_count * 16));
  if (stride == 4) kmeans_features_kernel<4><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, sel, n_sel, xf, feat);
  else kmeans_features_kernel<3><<<grid, 256, 0, s>>>(coords, n_frames, n_atoms, sel, n_sel, xf, feat);
  return cudaGetLastError();
}

cudaError_t kmeans_gather(const double* feat, int64_t nf, const int64_t* idx, int k, double* centers, cudaStream_t s) {
  kmeans_gather_kernel<<<k, 256, 0, s>>>(feat, nf, idx, centers);
  return cudaGetLastError();
}

cudaError_t kmeans_assign(const double* feat, int64_t n, int64_t nf, const double* centers, int k, int* labels,
                          double* dist_own, cudaStream_t s) {
  (void)dist_own;
  const unsigned g = (unsigned)((n + kAsRows - 1) / kAsRows);
  if (k <= kAsWarps)
    kmeans_assign_kernel<1><<<g, kAsWarps * 32, 0, s>>>(feat, n, nf, centers, k, labels, nullptr, nullptr, nullptr);
  else
    kmeans_assign_kernel<2><<<g, kAsWarps * 32, 0, s>>>(feat, n, nf, centers, k, labels, nullptr, nullptr, nullptr);
  return cudaGetLastError();
}

cudaError_t kmeans_sums(const double* feat, int64_t n, int64_t nf, const int* labels, int k, double* sums, int* counts,
                        cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kmeans_sums_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSumSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const dim3 grid((unsigned)((nf + kSumWarps * 32 - 1) / (kSumWarps * 32)), (unsigned)k);
  kmeans_sums_kernel<<<grid, kSumWarps * 32, kSumSmem, s>>>(feat, n, nf, labels, k, sums, counts);
  return cudaGetLastError();
}

cudaError_t kmeans_centers(const double* feat, int64_t nf, const double* sums, const int* counts, const int64_t* reseed,
                           int k, const double* old_c, double* new_c, double* shift, cudaStream_t s) {
  kmeans_centers_kernel<<<k, 256, 0, s>>>(feat, nf, sums, counts, reseed, old_c, new_c, shift);
  return cudaGetLastError();
}

cudaError_t kmeans_finish(const double* feat, int64_t n, int64_t nf, const double* centers, const int* labels, int k,
                          double* dist, unsigned long long* best_bits, unsigned* sizes, unsigned* centroids,
                          cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(sizes, 0, (size_t)k * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(centroids, 0xff, (size_t)k * sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(best_bits, 0xff, (size_t)k * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  const unsigned lin = (unsigned)((n + 127) / 128);
  sizes_kernel<<<lin, 128, 0, s>>>(labels, n, sizes);
  const unsigned g = (unsigned)((n + kAsRows - 1) / kAsRows);
  if (k <= kAsWarps)
    kmeans_assign_kernel<1><<<g, kAsWarps * 32, 0, s>>>(feat, n, nf, centers, k, nullptr, labels, dist, best_bits);
  else
    kmeans_assign_kernel<2><<<g, kAsWarps * 32, 0, s>>>(feat, n, nf, centers, k, nullptr, labels, dist, best_bits);
  medoid_pick_kernel<<<lin, 128, 0, s>>>(n, labels, dist, best_bits, centroids);
  return cudaGetLastError();
}

}  // namespace wmd

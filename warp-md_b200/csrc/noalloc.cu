// noalloc.cu -- wmd_rmsd_frames_noalloc: per-frame aligned RMSD for callers
// that cannot allocate memory.
//
// Who needs it: code that runs where allocating is not allowed or not safe --
// for example inside a host callback or a real-time loop that must not block
// on the allocator, a plugin that is handed device buffers by a host program
// that owns all GPU memory, or code that has no context object to keep
// workspaces in.  wmd_rmsd_frames needs a wmd_ctx and a wmd_ref, and both
// allocate (streams, events, a mapped status word, the centred reference and
// growable scratch).  This entry point takes only caller-owned device buffers
// and keeps its scratch in one fixed array compiled into the library.
//
// The scratch is a file-scope __device__ array of kScratchBytes (16 MiB).
// Every GPU that loads the library holds its own copy until the process exits.
// Host code cannot use the array's name as a device address, so the first
// call on each device (with that device current) looks the address up with
// cudaGetSymbolAddress and caches it; make that first call before any stream
// capture.  The cached address is not refreshed: after cudaDeviceReset (or
// anything else that replaces the device's primary context) it is stale, and
// the library must be reloaded before this entry point is used again on that
// device.  All calls on a device share the array and it keeps the last call's
// contents (each call clears what must start at zero): calls that may run at
// the same time on the GPU (different streams, or different host threads)
// race on it and must be serialised by the caller.
//
// A device-side wait that gives up (the streaming kernel's bounded mbarrier
// waits, 4 s) cannot be returned as an error code, because the call returns
// before the GPU runs and reading the status back would need a host
// synchronisation.  The kernels report it in the output instead: every frame
// of the affected batch is NaN.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/warpmd_rmsd.h"
#include "device_util.cuh"
#include "qcp.cuh"
#include "wmd_internal.h"

#define WMD_EXPORT extern "C" __attribute__((visibility("default")))

namespace wmd {
namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;     // the whole fixed array
constexpr int64_t kMaxAtoms = 65536;                    // largest selection accepted
constexpr size_t kHeaderBytes = 256;                    // reference statistics
constexpr size_t kYcOffset = kHeaderBytes;              // centred reference, FP64
constexpr size_t kYcBytes = (size_t)kMaxAtoms * 3 * sizeof(double);
constexpr size_t kWorkOffset = kYcOffset + kYcBytes;    // tile partials + refine records
constexpr size_t kWorkBytes = kScratchBytes - kWorkOffset;

// header layout (doubles): [0..2] mean(y), [3..5] sum of y_c, [6] G_y
constexpr int kHdrMean = 0, kHdrSumC = 3, kHdrGy = 6;
constexpr size_t kCountOffset = 128;   // unsigned: refine record count
constexpr size_t kStatusOffset = 132;  // int: device-side status bits

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::atomic<void*> g_scratch_addr[64] = {};  // per device, set on first use

// the message is read back with wmd_last_error(NULL)
int fail(int code, const char* msg) {
  set_thread_error(msg);
  return code;
}

// Reference statistics on the device (one CTA): mean, y_c = y - mean,
// sum of y_c and G_y, each reduced in a fixed tree order.
__global__ void __launch_bounds__(256) na_ref_prep(const float* __restrict__ ref, int64_t n, int stride,
                                                   unsigned char* __restrict__ scratch) {
  __shared__ double red[8][3];
  __shared__ double bc[4];
  double* hdr = reinterpret_cast<double*>(scratch);
  double* yc = reinterpret_cast<double*>(scratch + kYcOffset);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto block_sum3 = [&](double& a, double& b, double& c) {
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
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) {
    s0 += ref[k * stride + 0]; s1 += ref[k * stride + 1]; s2 += ref[k * stride + 2];
  }
  block_sum3(s0, s1, s2);
  const double inv = 1.0 / (double)n;
  const double m0 = s0 * inv, m1 = s1 * inv, m2 = s2 * inv;
  double c0 = 0, c1 = 0, c2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) {
    const double a = (double)ref[k * stride + 0] - m0;
    const double b = (double)ref[k * stride + 1] - m1;
    const double c = (double)ref[k * stride + 2] - m2;
    yc[k * 3 + 0] = a; yc[k * 3 + 1] = b; yc[k * 3 + 2] = c;
    c0 += a; c1 += b; c2 += c;
  }
  block_sum3(c0, c1, c2);
  double g0 = 0, g1 = 0, g2 = 0;
  for (int64_t k = tid; k < n; k += blockDim.x) {
    const double a = yc[k * 3 + 0] - c0 * inv, b = yc[k * 3 + 1] - c1 * inv, c = yc[k * 3 + 2] - c2 * inv;
    g0 += a * a; g1 += b * b; g2 += c * c;
  }
  block_sum3(g0, g1, g2);
  if (tid == 0) {
    hdr[kHdrMean + 0] = m0; hdr[kHdrMean + 1] = m1; hdr[kHdrMean + 2] = m2;
    hdr[kHdrSumC + 0] = c0; hdr[kHdrSumC + 1] = c1; hdr[kHdrSumC + 2] = c2;
    hdr[kHdrGy] = g0 + g1 + g2;
    *reinterpret_cast<unsigned*>(scratch + kCountOffset) = 0u;
  }
}

// One warp per frame: tile partials in tile order, then QCP; frames with
// near-zero RMSD are queued for the explicit residual pass.
__global__ void __launch_bounds__(256) na_finalize(const double* __restrict__ partial, int n_tiles, int64_t n_frames,
                                                   int64_t n_sel, unsigned char* __restrict__ scratch,
                                                   double* __restrict__ refine, double* __restrict__ out) {
  const int64_t f = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (f >= n_frames) return;
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  if (lane < 16) {
    const double* p = partial + (size_t)f * n_tiles * kStatDoubles + lane;
    for (int t = 0; t < n_tiles; ++t) s += p[(size_t)t * kStatDoubles];
  }
  double tot[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) tot[e] = __shfl_sync(0xffffffffu, s, e);
  if (lane != 0) return;
  if (*reinterpret_cast<const volatile int*>(scratch + kStatusOffset) != 0) {
    out[f] = __longlong_as_double(0x7ff8000000000000ll);  // the batch's partials are incomplete
    return;
  }
  const double* hdr = reinterpret_cast<const double*>(scratch);
  const double n = (double)n_sel, inv_n = 1.0 / n;
  const double sx[3] = {tot[0], tot[1], tot[2]};
  double h[9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) h[a * 3 + b] = tot[6 + a * 3 + b] - sx[a] * hdr[kHdrSumC + b] * inv_n;
  const double gx = tot[3] + tot[4] + tot[5] - (sx[0] * sx[0] + sx[1] * sx[1] + sx[2] * sx[2]) * inv_n;
  const double gy = hdr[kHdrGy];
  const QcpOut q = qcp_lambda(h, 0.5 * (gx + gy));
  const double rmsd = sqrt(msd_from(gx, gy, q.lambda, n));
  out[f] = rmsd;
  if (rmsd < kRefineScale * (gx + gy) * inv_n) {
    const unsigned slot = atomicAdd(reinterpret_cast<unsigned*>(scratch + kCountOffset), 1u);
    double* rec = refine + (size_t)slot * kStatDoubles;
    rec[0] = (double)f;
    rec[1] = sx[0] * inv_n; rec[2] = sx[1] * inv_n; rec[3] = sx[2] * inv_n;
    for (int e = 0; e < 9; ++e) rec[4 + e] = h[e];
    rec[13] = q.lambda;
  }
}

// Explicit FP64 residuals for the queued frames (one CTA per frame).
__global__ void __launch_bounds__(256) na_refine(const float* __restrict__ coords, int64_t n_atoms, int stride,
                                                 int64_t n_sel, const unsigned char* __restrict__ scratch,
                                                 const double* __restrict__ refine, double* __restrict__ out) {
  __shared__ double sh[12];
  __shared__ double red[8];
  const unsigned count = *reinterpret_cast<const unsigned*>(scratch + kCountOffset);
  const double* hdr = reinterpret_cast<const double*>(scratch);
  const double* yc = reinterpret_cast<const double*>(scratch + kYcOffset);
  const double inv_n = 1.0 / (double)n_sel;
  const double my0 = hdr[kHdrSumC] * inv_n, my1 = hdr[kHdrSumC + 1] * inv_n, my2 = hdr[kHdrSumC + 2] * inv_n;
  for (unsigned r = blockIdx.x; r < count; r += gridDim.x) {
    const double* rec = refine + (size_t)r * kStatDoubles;
    if (threadIdx.x == 0) {
      double h[9], R[9];
      for (int e = 0; e < 9; ++e) h[e] = rec[4 + e];
      rotation_from_qcp(h, rec[13], R);
      for (int e = 0; e < 9; ++e) sh[e] = R[e];
      sh[9] = rec[1]; sh[10] = rec[2]; sh[11] = rec[3];
    }
    __syncthreads();
    const int64_t f = (int64_t)rec[0];
    const float* frame = coords + (size_t)f * n_atoms * stride;
    double acc = 0.0;
    for (int64_t k = threadIdx.x; k < n_sel; k += blockDim.x) {
      const float* p = frame + k * stride;
      const double d0 = (double)p[0] - sh[9], d1 = (double)p[1] - sh[10], d2 = (double)p[2] - sh[11];
      const double r0 = sh[0] * d0 + sh[1] * d1 + sh[2] * d2 - (yc[k * 3 + 0] - my0);
      const double r1 = sh[3] * d0 + sh[4] * d1 + sh[5] * d2 - (yc[k * 3 + 1] - my1);
      const double r2 = sh[6] * d0 + sh[7] * d1 + sh[8] * d2 - (yc[k * 3 + 2] - my2);
      acc += r0 * r0 + r1 * r1 + r2 * r2;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += red[w];
      out[f] = sqrt(t * inv_n);
    }
    __syncthreads();
  }
}

// Device (or managed) memory that the current device can address without
// peer access: a buffer of another GPU would be an illegal address here.
bool is_device_here(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace
}  // namespace wmd

// Per-frame aligned RMSD (the same result as wmd_rmsd_frames with align = 1
// and a dense selection) using only the library's fixed scratch array.  See
// include/warpmd_rmsd.h for the contract.
WMD_EXPORT int wmd_rmsd_frames_noalloc(const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                       const float* ref, int64_t n_sel, int ref_stride, double* out, void* stream) {
  using namespace wmd;
  if (stride != 3 && stride != 4) return fail(WMD_ERR_INVALID_ARG, "stride must be 3 or 4");
  if (ref_stride != 3 && ref_stride != 4) return fail(WMD_ERR_INVALID_ARG, "ref_stride must be 3 or 4");
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return fail(WMD_ERR_INVALID_ARG, "negative size");
  if (n_sel > n_atoms) return fail(WMD_ERR_MISMATCH, "selection exceeds the frame's atom count");
  if (n_sel > kMaxAtoms) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "wmd_rmsd_frames_noalloc accepts at most %lld selected atoms (got %lld); use wmd_rmsd_frames",
             (long long)kMaxAtoms, (long long)n_sel);
    return fail(WMD_ERR_INVALID_ARG, msg);
  }
  if (n_frames == 0) return WMD_OK;
  if (!coords || !out || (n_sel > 0 && !ref)) return fail(WMD_ERR_INVALID_ARG, "null pointer");
  cudaError_t e;
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess || dev < 0 || dev >= 64) return fail(WMD_ERR_CUDA, "no current device");
  if (!is_device_here(coords, dev) || !is_device_here(out, dev) || (n_sel > 0 && !is_device_here(ref, dev)))
    return fail(WMD_ERR_INVALID_ARG, "coords, ref and out must be device memory of the current device");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_sel == 0) {
    e = cudaMemsetAsync(out, 0, (size_t)n_frames * sizeof(double), s);
    return e == cudaSuccess ? WMD_OK : fail(WMD_ERR_CUDA, cudaGetErrorString(e));
  }
  int major = 0, sms = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (major != 10) return fail(WMD_ERR_NO_DEVICE, "current device is not an sm_100 (B200) device");
  void* addr = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!addr) {
    // every thread that races here looks up the same address
    if ((e = cudaGetSymbolAddress(&addr, g_noalloc_scratch)) != cudaSuccess || !addr)
      return fail(WMD_ERR_CUDA, e == cudaSuccess ? "scratch address lookup returned null" : cudaGetErrorString(e));
    g_scratch_addr[dev].store(addr, std::memory_order_release);
  }
  unsigned char* scratch = static_cast<unsigned char*>(addr);

  na_ref_prep<<<1, 256, 0, s>>>(ref, n_sel, ref_stride, scratch);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(WMD_ERR_CUDA, cudaGetErrorString(e));

  FrameLaunch L;
  L.n_atoms = n_atoms;
  L.stride = stride;
  L.gather = (reinterpret_cast<uintptr_t>(coords) & 15u) != 0;
  L.tile_atoms = kConsumerThreads * 8;
  L.align = 1;
  L.ref.yc = reinterpret_cast<const double*>(scratch + kYcOffset);
  L.ref.n_sel = n_sel;
  L.status = reinterpret_cast<int*>(scratch + kStatusOffset);
  const int tiles = frame_tiles(L);
  // Frames per launch so that partials and refine records fit the work area,
  // a multiple of 4 so that each batch's first frame keeps the 16-byte
  // alignment of `coords` (4 frames of stride-3 floats are 48 n_atoms bytes).
  const size_t per_frame = (size_t)(tiles + 1) * kStatDoubles * sizeof(double);
  int64_t batch = std::max<int64_t>(1, std::min<int64_t>(n_frames, (int64_t)(kWorkBytes / per_frame)));
  if (batch < n_frames && batch >= 4) batch &= ~int64_t(3);
  double* partial = reinterpret_cast<double*>(scratch + kWorkOffset);
  double* refine = partial + (size_t)batch * tiles * kStatDoubles;
  for (int64_t f0 = 0; f0 < n_frames; f0 += batch) {
    const int64_t nf = std::min(batch, n_frames - f0);
    FrameLaunch B = L;
    B.coords = coords + (size_t)f0 * n_atoms * stride;
    // the staged kernel bulk-copies from 16-byte boundaries of its base
    B.gather = (reinterpret_cast<uintptr_t>(B.coords) & 15u) != 0;
    B.n_frames = nf;
    B.partial = partial;
    B.grid = frame_grid(B, sms, false);
    // refine count and status word start at zero for every batch
    static_assert(kStatusOffset == kCountOffset + sizeof(unsigned), "count and status are adjacent");
    if ((e = cudaMemsetAsync(scratch + kCountOffset, 0, sizeof(unsigned) + sizeof(int), s)) != cudaSuccess)
      return fail(WMD_ERR_CUDA, cudaGetErrorString(e));
    if ((e = launch_rmsd_stream(B, s)) != cudaSuccess) return fail(WMD_ERR_CUDA, cudaGetErrorString(e));
    na_finalize<<<(unsigned)((nf + 7) / 8), 256, 0, s>>>(partial, tiles, nf, n_sel, scratch, refine, out + f0);
    na_refine<<<(unsigned)std::min<int64_t>(nf, 148), 256, 0, s>>>(B.coords, n_atoms, stride, n_sel, scratch, refine,
                                                                    out + f0);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(WMD_ERR_CUDA, cudaGetErrorString(e));
  }
  return WMD_OK;
}

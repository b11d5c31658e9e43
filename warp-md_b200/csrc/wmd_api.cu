// wmd_api.cu -- host side of libwarpmd_rmsd.so: the C ABI declared in
// include/warpmd_rmsd.h.
//
// Plays the role of the reference's GpuContext (crates/traj-gpu/src/cuda.rs,
// crates/traj-gpu/src/cuda/runtime_core.rs:375-535) without runtime
// compilation: kernels are built ahead of time for sm_100a.  Differences by
// design:
//   * host inputs are streamed in chunks through two device buffers, with the
//     host->device copy of chunk k+1 (copy stream) overlapping the kernel of
//     chunk k (caller's stream), instead of one synchronous clone_htod per
//     chunk followed by three synchronous downloads;
//   * the reference is centred once, in FP64, at upload time;
//   * the per-frame QCP runs on the device in the same launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <memory>
#include <thread>
#include <vector>

#include "../../include/warpmd_rmsd.h"
#include "batched.h"
#include "cluster.h"
#include "dcd.h"
#include "device_util.cuh"
#include "fluct.h"
#include "pairwise.h"
#include "pairwise_dme.h"
#include "superpose.h"
#include "wmd_internal.h"

#define WMD_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

constexpr const char* kVersion = "0.4.30+b200.1";
// Host-input chunk size for the streaming pipeline.
constexpr size_t kChunkBytes = size_t(256) << 20;
// Scratch bound for one forward launch's tile partials.
constexpr size_t kPartialBytesMax = size_t(512) << 20;

thread_local std::string g_create_error;

// Compensated summation (Neumaier 1974): error bounded by ~2 eps |sum| plus
// O(n eps^2) sum |x_i|, independent of the order of magnitudes.
struct NeumaierSum {
  double s = 0.0, c = 0.0;
  void add(double x) {
    const double t = s + x;
    if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

struct HostBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct wmd_ref {
  double* yc = nullptr;
  float* w = nullptr;  // per-atom weights (weighted references only)
  wmd::RefInfo info;
};

struct wmd_group_ref {
  void* mem = nullptr;  // one allocation: offsets, atoms, blocks, reference
  uint32_t* goff = nullptr;
  uint32_t* gatoms = nullptr;
  uint32_t* blocks = nullptr;
  float* ref_all = nullptr;
  int64_t n_atoms = 0, n_groups = 0, n_blocks = 0;
  int64_t contig_base = -1;  // >= 0 when group_atoms[q] == contig_base + q
};

struct wmd_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t h2d_done[2] = {nullptr, nullptr};
  cudaEvent_t kern_done[2] = {nullptr, nullptr};
  int* status_host = nullptr;  // mapped pinned word the kernels report into
  int* status_dev = nullptr;
  wmd::WaitCfg wait;           // bounded-wait limits (wmd_set_wait_test)
  DevBuf partial, refine, refine_count, rot, chunk[2], out_tmp, sel_buf, aux, out_chunk;
  DevBuf fl_part, fl_acc, fl_shift;
  DevBuf vg_stats;  // frame records of wmd_rmsd_value_and_grad's two-kernel route
  DevBuf cl_mat, cl_scratch, cl_out, km_feat, km_xf, km_work;  // clustering  // fluctuations, per-group RMSD
  // a sorted host selection expanded onto its atom span for the
  // frames-across-lanes kernel, valid for the current call
  DevBuf lane_exp;
  struct {
    bool valid = false;
    int64_t a0 = 0, span = 0;
    const double* y = nullptr;
    const float* w = nullptr;
  } lx;
  HostBuf stage[2];
  std::string err;
  wmd::PairwiseWorkspace pw;
  // batched launch prepared by wmd_batched_prepare
  DevBuf b_segs, b_yc, b_partial, b_rot, b_refine, b_count, b_maps;
  std::vector<wmd_batch_desc> b_descs;
  bool b_grad = false;
  bool b_ready = false;
  wmd::BatchPlan b_plan;
};

namespace {

int set_err(wmd_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  else g_create_error = buf;
  return code;
}

int cuda_err(wmd_ctx* ctx, cudaError_t e, const char* what) {
  // same wording as the reference's map_driver_err (crates/traj-gpu/src/cuda.rs:384-386)
  return set_err(ctx, e == cudaErrorMemoryAllocation ? WMD_ERR_OOM : WMD_ERR_CUDA, "cuda driver error: %s: %s",
                 what, cudaGetErrorString(e));
}

#define CU(call, what)                                  \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_err(ctx, _e, what); \
  } while (0)

// Keeps the caller's current device across a call.
// Makes `dev` current for the call and restores the caller's device.  The
// device is set even when it already is the thread's device: cudaSetDevice
// also makes its primary context current on this thread, which driver-API
// calls (the tensor-map encodes) need on threads where no runtime call has
// bound it yet, such as the autograd engine's worker threads.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

enum class Mem { Null, Device, PinnedHost, PageableHost };

Mem classify(const void* p) {
  if (!p) return Mem::Null;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return Mem::PageableHost;
  }
  switch (a.type) {
    case cudaMemoryTypeDevice:
    case cudaMemoryTypeManaged:
      return Mem::Device;
    case cudaMemoryTypeHost:
      return Mem::PinnedHost;
    default:
      return Mem::PageableHost;
  }
}

bool is_host(Mem m) { return m == Mem::PinnedHost || m == Mem::PageableHost; }

int ensure(wmd_ctx* ctx, DevBuf& b, size_t bytes, bool zero = false) {
  if (b.bytes >= bytes && b.ptr) return WMD_OK;
  if (b.ptr) {
    cudaFree(b.ptr);  // synchronizes the device: no launch still uses it
    b.ptr = nullptr;
    b.bytes = 0;
  }
  size_t want = std::max<size_t>(bytes, 256);
  cudaError_t e = cudaMalloc(&b.ptr, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.ptr = nullptr;
    return set_err(ctx, WMD_ERR_OOM, "cuda driver error: device allocation of %zu bytes failed: %s", want,
                   cudaGetErrorString(e));
  }
  b.bytes = want;
  if (zero) {
    e = cudaMemset(b.ptr, 0, want);
    if (e != cudaSuccess) return cuda_err(ctx, e, "cudaMemset");
  }
  return WMD_OK;
}

int ensure_host(wmd_ctx* ctx, HostBuf& b, size_t bytes) {
  if (b.bytes >= bytes && b.ptr) return WMD_OK;
  if (b.ptr) {
    cudaFreeHost(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
  }
  cudaError_t e = cudaHostAlloc(&b.ptr, bytes, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.ptr = nullptr;
    return set_err(ctx, WMD_ERR_OOM, "pinned host allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  }
  b.bytes = bytes;
  return WMD_OK;
}

// Reports timeouts / bad indices recorded by earlier kernels.
int check_status(wmd_ctx* ctx) {
  const int st = __atomic_exchange_n(ctx->status_host, 0, __ATOMIC_ACQ_REL);
  if (st == 0) return WMD_OK;
  if (st & 16) return set_err(ctx, WMD_ERR_INVALID_ARG, "selection index out of range (status 0x%x)", st);
  return set_err(ctx, WMD_ERR_TIMEOUT, "a device-side wait exceeded its limit (status 0x%x)", st);
}

int check_common(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                 const uint32_t* sel, int64_t n_sel, const wmd_ref* ref) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!ref) return set_err(ctx, WMD_ERR_INVALID_ARG, "reference is null");
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_frames > 0 && !coords) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords is null");
  if (ref->info.w)
    return set_err(ctx, WMD_ERR_INVALID_ARG, "a weighted reference serves the superposition entry points only");
  if (n_sel != ref->info.n_sel)
    return set_err(ctx, WMD_ERR_MISMATCH, "reference has %lld atoms but the selection has %lld",
                   (long long)ref->info.n_sel, (long long)n_sel);
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  return WMD_OK;
}

// Resolves the selection to a device pointer, validating host indices.
int resolve_sel(wmd_ctx* ctx, const uint32_t* sel, int64_t n_sel, int64_t n_atoms, const uint32_t** dsel,
                cudaStream_t s) {
  *dsel = nullptr;
  if (!sel) return WMD_OK;
  const Mem m = classify(sel);
  if (m == Mem::Device) {
    *dsel = sel;
    return WMD_OK;
  }
  for (int64_t i = 0; i < n_sel; ++i)
    if ((int64_t)sel[i] >= n_atoms)
      return set_err(ctx, WMD_ERR_INVALID_ARG, "selection index %u out of range for %lld atoms", sel[i],
                     (long long)n_atoms);
  int rc = ensure(ctx, ctx->sel_buf, (size_t)n_sel * 4);
  if (rc) return rc;
  CU(cudaMemcpyAsync(ctx->sel_buf.ptr, sel, (size_t)n_sel * 4, cudaMemcpyHostToDevice, s), "upload selection");
  *dsel = static_cast<const uint32_t*>(ctx->sel_buf.ptr);
  return WMD_OK;
}

// A host selection that is strictly increasing and at least 1/4 dense is
// streamed by the frames-across-lanes kernel as the atom span it covers: the
// reference (centred, weighted) and the weights are expanded onto the span,
// unselected atoms weighing 0.  At that density the gathered loads fetch
// most sectors of the span anyway, at a latency-bound rate; the span streams
// at the HBM rate.  Sparser selections (1 in 10: the gathered loads fetch
// about half the span's sectors) stay on the gathered path, which measured
// faster there.  Valid for the current call (LaneScope).
int lanes_prepare(wmd_ctx* ctx, const uint32_t* sel, const uint32_t* dsel, int64_t n_sel, int stride,
                  const wmd_ref* ref, cudaStream_t s) {
  ctx->lx.valid = false;
  if (!sel || !dsel || n_sel < 64 || !is_host(classify(sel))) return WMD_OK;
  for (int64_t i = 1; i < n_sel; ++i)
    if (sel[i] <= sel[i - 1]) return WMD_OK;
  const int64_t a0 = stride == 4 ? (int64_t)sel[0] : (int64_t)(sel[0] & ~3u);  // 16-byte aligned first atom
  const int64_t span = (int64_t)sel[n_sel - 1] + 1 - a0;
  if (span > 4 * n_sel) return WMD_OK;
  const size_t ybytes = ((size_t)(span + 32) * 3 * sizeof(double) + 255) & ~size_t(255);
  const size_t wbytes = (size_t)(span + 32) * sizeof(float);
  int rc = ensure(ctx, ctx->lane_exp, ybytes + wbytes);
  if (rc) return rc;
  double* y = static_cast<double*>(ctx->lane_exp.ptr);
  float* w = reinterpret_cast<float*>(static_cast<char*>(ctx->lane_exp.ptr) + ybytes);
  CU(cudaMemsetAsync(ctx->lane_exp.ptr, 0, ybytes + wbytes, s), "memset");
  CU(wmd::launch_lanes_expand(dsel, n_sel, a0, ref->yc, ref->info.w, y, w, s), "selection expansion");
  ctx->lx.valid = true;
  ctx->lx.a0 = a0;
  ctx->lx.span = span;
  ctx->lx.y = y;
  ctx->lx.w = w;
  return WMD_OK;
}

struct LaneScope {
  wmd_ctx* ctx;
  ~LaneScope() { ctx->lx.valid = false; }
};

// The expansion of the current call, if any, for launches over `dsel`.
void apply_lanes(wmd_ctx* ctx, wmd::FrameLaunch& L, const uint32_t* dsel) {
  if (!dsel || !ctx->lx.valid) return;
  L.lane_atom0 = ctx->lx.a0;
  L.lane_atoms = ctx->lx.span;
  L.lane_y = ctx->lx.y;
  L.lane_w = ctx->lx.w;
}

wmd::FrameLaunch base_launch(wmd_ctx* ctx, const wmd_ref* ref, int64_t n_atoms, int stride, const uint32_t* dsel) {
  wmd::FrameLaunch L;
  L.n_atoms = n_atoms;
  L.stride = stride;
  L.sel = dsel;
  L.ref = ref->info;
  L.ref.yc = ref->yc;
  L.status = ctx->status_dev;
  L.wait = ctx->wait;
  L.tile_atoms = wmd::kConsumerThreads * 8;
  return L;
}

wmd::VgLaunch vg_launch(wmd_ctx* ctx, const wmd_ref* ref, const float* coords, int64_t n_frames, int64_t n_atoms) {
  wmd::VgLaunch V;
  V.coords = coords;
  V.n_frames = n_frames;
  V.n_atoms = n_atoms;
  V.ref = ref->info;
  V.ref.yc = ref->yc;
  V.status = ctx->status_dev;
  V.wait = ctx->wait;
  return V;
}

// Frames per batch when at most `fit` fit the scratch: a multiple of 4 when the
// frames are split, so that every batch starts at the 16-byte alignment of
// frame 0 (4 frames of float32 atoms are a multiple of 16 bytes).
int64_t frame_batch(size_t fit, int64_t n_frames) {
  int64_t b = std::max<int64_t>(1, (int64_t)std::min<size_t>(fit, (size_t)INT64_MAX));
  if (b >= n_frames) return n_frames;
  return b >= 4 ? (b & ~int64_t(3)) : b;
}

// The staged atom-major kernel bulk-copies from 16-byte boundaries of its base:
// a batch whose first frame is not 16-byte aligned runs the gathered kernel
// (same tiles, same partials).  The frames-across-lanes kernel needs no check:
// it only runs when the frame stride is a multiple of 16 bytes.
void keep_aligned(wmd::FrameLaunch& B) {
  if (!B.lanes && !B.gather && (reinterpret_cast<uintptr_t>(B.coords) & 15u) != 0) B.gather = true;
}

// Runs the forward over device-resident frames, splitting into frame batches
// so the tile-partial scratch stays bounded.  `o` points at frame 0 outputs.
int forward_device(wmd_ctx* ctx, const float* dcoords, int64_t n_frames, int64_t n_atoms, int stride,
                   const uint32_t* dsel, const wmd_ref* ref, int align, wmd::FrameOutputs o, cudaStream_t s) {
  if (n_frames == 0) return WMD_OK;
  wmd::FrameLaunch L = base_launch(ctx, ref, n_atoms, stride, dsel);
  L.align = align;
  L.gather = dsel != nullptr || (reinterpret_cast<uintptr_t>(dcoords) & 15u) != 0;
  L.coords = dcoords;
  L.n_frames = n_frames;
  apply_lanes(ctx, L, dsel);
  wmd::frame_plan(L, ctx->sm_count);
  const int tiles = wmd::frame_tiles(L);
  const size_t per_frame = (size_t)tiles * wmd::kStatDoubles * sizeof(double);
  const int64_t batch = frame_batch(kPartialBytesMax / per_frame, n_frames);
  {
    int rc = ensure(ctx, ctx->partial, per_frame * (size_t)batch);
    if (rc) return rc;
  }
  if (align) {
    int rc = ensure(ctx, ctx->refine, (size_t)batch * wmd::kStatDoubles * sizeof(double));
    if (rc) return rc;
    rc = ensure(ctx, ctx->refine_count, sizeof(unsigned), true);
    if (rc) return rc;
  }
  for (int64_t f0 = 0; f0 < n_frames; f0 += batch) {
    const int64_t nf = std::min(batch, n_frames - f0);
    wmd::FrameLaunch B = L;
    if (align) {
      B.refine = static_cast<double*>(ctx->refine.ptr);
      B.refine_count = static_cast<unsigned*>(ctx->refine_count.ptr);
    }
    B.coords = dcoords + (size_t)f0 * n_atoms * stride;
    keep_aligned(B);
    B.n_frames = nf;
    B.out.rmsd = o.rmsd ? o.rmsd + f0 : nullptr;
    B.out.stats = o.stats ? o.stats + f0 * wmd::kStatDoubles : nullptr;
    B.out.cov = o.cov ? o.cov + f0 * 9 : nullptr;
    B.out.sum_x2 = o.sum_x2 ? o.sum_x2 + f0 : nullptr;
    B.out.sum_y2 = o.sum_y2 ? o.sum_y2 + f0 : nullptr;
    B.partial = static_cast<double*>(ctx->partial.ptr);
    B.grid = wmd::frame_grid(B, ctx->sm_count, false);
    CU(wmd::launch_rmsd_forward(B, s), "rmsd forward launch");
  }
  return WMD_OK;
}

// Host-resident frames: chunked double-buffered H2D overlapping the kernels.
int forward_host(wmd_ctx* ctx, const float* hcoords, Mem kind, int64_t n_frames, int64_t n_atoms, int stride,
                 const uint32_t* dsel, const wmd_ref* ref, int align, wmd::FrameOutputs o, cudaStream_t s) {
  const size_t frame_bytes = (size_t)n_atoms * stride * sizeof(float);
  if (frame_bytes == 0) return forward_device(ctx, nullptr, 0, n_atoms, stride, dsel, ref, align, o, s);
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_frames, (int64_t)(kChunkBytes / frame_bytes)));
  const size_t chunk_bytes = (size_t)chunk * frame_bytes;
  for (int b = 0; b < 2; ++b) {
    int rc = ensure(ctx, ctx->chunk[b], chunk_bytes);
    if (rc) return rc;
    if (kind == Mem::PageableHost) {
      rc = ensure_host(ctx, ctx->stage[b], chunk_bytes);
      if (rc) return rc;
    }
  }
  // the buffers may have been used by earlier work on other streams
  CU(cudaEventRecord(ctx->kern_done[0], s), "event");
  CU(cudaEventRecord(ctx->kern_done[1], s), "event");
  CU(cudaEventRecord(ctx->h2d_done[0], ctx->copy_stream), "event");
  CU(cudaEventRecord(ctx->h2d_done[1], ctx->copy_stream), "event");
  int64_t k = 0;
  for (int64_t f0 = 0; f0 < n_frames; f0 += chunk, ++k) {
    const int b = (int)(k & 1);
    const int64_t nf = std::min(chunk, n_frames - f0);
    const size_t bytes = (size_t)nf * frame_bytes;
    const char* src = reinterpret_cast<const char*>(hcoords) + (size_t)f0 * frame_bytes;
    if (kind == Mem::PageableHost) {
      CU(cudaEventSynchronize(ctx->h2d_done[b]), "staging wait");
      std::memcpy(ctx->stage[b].ptr, src, bytes);
      src = static_cast<const char*>(ctx->stage[b].ptr);
    }
    CU(cudaStreamWaitEvent(ctx->copy_stream, ctx->kern_done[b], 0), "stream wait");
    CU(cudaMemcpyAsync(ctx->chunk[b].ptr, src, bytes, cudaMemcpyHostToDevice, ctx->copy_stream), "H2D");
    CU(cudaEventRecord(ctx->h2d_done[b], ctx->copy_stream), "event");
    CU(cudaStreamWaitEvent(s, ctx->h2d_done[b], 0), "stream wait");
    wmd::FrameOutputs oc;
    oc.rmsd = o.rmsd ? o.rmsd + f0 : nullptr;
    oc.stats = o.stats ? o.stats + f0 * wmd::kStatDoubles : nullptr;
    oc.cov = o.cov ? o.cov + f0 * 9 : nullptr;
    oc.sum_x2 = o.sum_x2 ? o.sum_x2 + f0 : nullptr;
    oc.sum_y2 = o.sum_y2 ? o.sum_y2 + f0 : nullptr;
    int rc = forward_device(ctx, static_cast<const float*>(ctx->chunk[b].ptr), nf, n_atoms, stride, dsel, ref, align,
                            oc, s);
    if (rc) return rc;
    CU(cudaEventRecord(ctx->kern_done[b], s), "event");
  }
  return WMD_OK;
}

}  // namespace

void wmd::set_thread_error(const char* msg) { g_create_error = msg; }

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

WMD_EXPORT const char* wmd_version(void) { return kVersion; }

WMD_EXPORT const char* wmd_last_error(const wmd_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

WMD_EXPORT int wmd_create(int device, wmd_ctx** out) {
  if (!out) return set_err(nullptr, WMD_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_err(nullptr, WMD_ERR_NO_DEVICE, "no CUDA device available (%s)",
                   e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
  }
  if (device < 0 || device >= n)
    return set_err(nullptr, WMD_ERR_INVALID_ARG, "invalid cuda device index %d (have %d)", device, n);
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess)
    return set_err(nullptr, WMD_ERR_CUDA, "cuda driver error: %s", cudaGetErrorString(e));
  if (prop.major != 10)
    return set_err(nullptr, WMD_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a (B200)", device,
                   prop.major, prop.minor);
  DeviceGuard g(device);
  wmd_ctx* ctx = new wmd_ctx();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  auto fail = [&](cudaError_t ee, const char* what) {
    std::string msg = std::string("cuda driver error: ") + what + ": " + cudaGetErrorString(ee);
    wmd_destroy(ctx);
    return set_err(nullptr, WMD_ERR_CUDA, "%s", msg.c_str());
  };
  if ((e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(e, "stream");
  for (int b = 0; b < 2; ++b) {
    if ((e = cudaEventCreateWithFlags(&ctx->h2d_done[b], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreateWithFlags(&ctx->kern_done[b], cudaEventDisableTiming)) != cudaSuccess)
      return fail(e, "event");
  }
  if ((e = cudaHostAlloc(&ctx->status_host, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable)) != cudaSuccess)
    return fail(e, "status word");
  *ctx->status_host = 0;
  if ((e = cudaHostGetDevicePointer(&ctx->status_dev, ctx->status_host, 0)) != cudaSuccess) return fail(e, "status word");
  *out = ctx;
  return WMD_OK;
}

WMD_EXPORT int wmd_destroy(wmd_ctx* ctx) {
  if (!ctx) return WMD_OK;
  DeviceGuard g(ctx->device);
  cudaDeviceSynchronize();
  for (DevBuf* b : {&ctx->partial, &ctx->refine, &ctx->refine_count, &ctx->rot, &ctx->chunk[0], &ctx->chunk[1], &ctx->out_tmp,
                    &ctx->sel_buf, &ctx->aux, &ctx->out_chunk, &ctx->fl_part, &ctx->fl_acc, &ctx->fl_shift, &ctx->cl_mat, &ctx->cl_scratch,
                    &ctx->cl_out, &ctx->km_feat, &ctx->km_xf, &ctx->km_work, &ctx->lane_exp, &ctx->vg_stats, &ctx->b_segs, &ctx->b_maps, &ctx->b_yc, &ctx->b_partial, &ctx->b_rot,
                    &ctx->b_refine, &ctx->b_count})
    if (b->ptr) cudaFree(b->ptr);
  for (HostBuf* b : {&ctx->stage[0], &ctx->stage[1]})
    if (b->ptr) cudaFreeHost(b->ptr);
  wmd::pairwise_workspace_free(ctx->pw);
  for (int b = 0; b < 2; ++b) {
    if (ctx->h2d_done[b]) cudaEventDestroy(ctx->h2d_done[b]);
    if (ctx->kern_done[b]) cudaEventDestroy(ctx->kern_done[b]);
  }
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->status_host) cudaFreeHost(ctx->status_host);
  delete ctx;
  return WMD_OK;
}

static int reference_upload(wmd_ctx* ctx, const float* ref, int64_t n_sel, int stride, const float* weights,
                            wmd_ref** out) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!out) return set_err(ctx, WMD_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_sel > 0 && !ref) return set_err(ctx, WMD_ERR_INVALID_ARG, "reference is null");
  DeviceGuard g(ctx->device);
  std::vector<float> host, hw;
  const float* h = ref;
  if (n_sel > 0 && classify(ref) == Mem::Device) {
    host.resize((size_t)n_sel * stride);
    CU(cudaMemcpy(host.data(), ref, host.size() * sizeof(float), cudaMemcpyDeviceToHost), "download reference");
    h = host.data();
  }
  const float* wt = weights;
  if (weights && n_sel > 0 && classify(weights) == Mem::Device) {
    hw.resize((size_t)n_sel);
    CU(cudaMemcpy(hw.data(), weights, hw.size() * sizeof(float), cudaMemcpyDeviceToHost), "download weights");
    wt = hw.data();
  }
  wmd_ref* r = new wmd_ref();
  wmd::RefInfo& I = r->info;
  I.n_sel = n_sel;
  I.wsum = (double)n_sel;
  std::vector<double> yc((size_t)std::max<int64_t>(n_sel, 1) * 3, 0.0);
  if (n_sel > 0 && !weights) {
    // FP64 two-pass centring, as rmsd_aligned_selected does (plan.rs:1172-1190).
    // The sums run over up to ~1e5 atoms whose coordinates are far from the
    // origin, so they are compensated (Neumaier): the kernels correct H with
    // sum(y_c) and must see the exact sum of the stored centred values.
    NeumaierSum m[3];
    for (int64_t i = 0; i < n_sel; ++i)
      for (int c = 0; c < 3; ++c) m[c].add((double)h[i * stride + c]);
    for (int c = 0; c < 3; ++c) I.mean[c] = m[c].value() / (double)n_sel;
    NeumaierSum sc[3], sq;
    for (int64_t i = 0; i < n_sel; ++i)
      for (int c = 0; c < 3; ++c) {
        const double y = (double)h[i * stride + c];
        yc[i * 3 + c] = y - I.mean[c];
        sc[c].add(yc[i * 3 + c]);
        sq.add(y * y);
      }
    for (int c = 0; c < 3; ++c) I.sum_c[c] = sc[c].value();
    I.sumsq = sq.value();
    NeumaierSum gy;
    for (int64_t i = 0; i < n_sel; ++i)
      for (int c = 0; c < 3; ++c) {
        const double d = yc[i * 3 + c] - I.sum_c[c] / (double)n_sel;
        gy.add(d * d);
      }
    I.gy = gy.value();
  } else if (n_sel > 0) {
    // weighted (centroid_weighted / kabsch_rotation_weighted,
    // geometry_math.rs:202-300): mean_w = sum w y / sum w; the stored rows
    // are w (y - mean_w), sum_c their exact sum, G_y = sum w |y - mean_w|^2
    NeumaierSum ws, m[3];
    for (int64_t i = 0; i < n_sel; ++i) {
      const double w = (double)wt[i];
      ws.add(w);
      for (int c = 0; c < 3; ++c) m[c].add(w * (double)h[i * stride + c]);
    }
    I.wsum = ws.value();
    for (int c = 0; c < 3; ++c) I.mean[c] = I.wsum != 0.0 ? m[c].value() / I.wsum : 0.0;
    NeumaierSum sc[3], sq;
    std::vector<double> d((size_t)n_sel * 3);
    for (int64_t i = 0; i < n_sel; ++i)
      for (int c = 0; c < 3; ++c) {
        const double y = (double)h[i * stride + c];
        d[i * 3 + c] = y - I.mean[c];
        yc[i * 3 + c] = (double)wt[i] * d[i * 3 + c];
        sc[c].add(yc[i * 3 + c]);
        sq.add((double)wt[i] * y * y);
      }
    for (int c = 0; c < 3; ++c) I.sum_c[c] = sc[c].value();
    I.sumsq = sq.value();
    NeumaierSum gy;
    for (int64_t i = 0; i < n_sel; ++i)
      for (int c = 0; c < 3; ++c) {
        const double e = d[i * 3 + c] - (I.wsum != 0.0 ? I.sum_c[c] / I.wsum : 0.0);
        gy.add((double)wt[i] * e * e);
      }
    I.gy = gy.value();
  }
  // 32 zero atoms after the reference: the frames-across-lanes kernel copies
  // whole 32-atom blocks of it
  const size_t yc_pad = 32 * 3;
  cudaError_t e = cudaMalloc(&r->yc, (yc.size() + yc_pad) * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(r->yc + yc.size(), 0, yc_pad * sizeof(double));
  if (e == cudaSuccess && weights && n_sel > 0) {
    e = cudaMalloc(&r->w, (size_t)(n_sel + 32) * sizeof(float));  // + 32 zero weights, as yc
    if (e == cudaSuccess) e = cudaMemset(r->w + n_sel, 0, 32 * sizeof(float));
  }
  if (e != cudaSuccess) {
    cudaFree(r->yc);
    delete r;
    cudaGetLastError();
    return set_err(ctx, WMD_ERR_OOM, "cuda driver error: reference allocation failed: %s", cudaGetErrorString(e));
  }
  e = cudaMemcpy(r->yc, yc.data(), yc.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && r->w) e = cudaMemcpy(r->w, wt, (size_t)n_sel * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(r->yc);
    cudaFree(r->w);
    delete r;
    return cuda_err(ctx, e, "upload reference");
  }
  I.yc = r->yc;
  I.w = r->w;
  *out = r;
  return WMD_OK;
}

WMD_EXPORT int wmd_reference_upload(wmd_ctx* ctx, const float* ref, int64_t n_sel, int stride, wmd_ref** out) {
  return reference_upload(ctx, ref, n_sel, stride, nullptr, out);
}

WMD_EXPORT int wmd_reference_upload_weighted(wmd_ctx* ctx, const float* ref, int64_t n_sel, int stride,
                                             const float* weights, wmd_ref** out) {
  return reference_upload(ctx, ref, n_sel, stride, weights, out);
}

WMD_EXPORT int wmd_reference_free(wmd_ctx* ctx, wmd_ref* ref) {
  if (!ref) return WMD_OK;
  if (ctx) {
    DeviceGuard g(ctx->device);
    cudaFree(ref->yc);
    if (ref->w) cudaFree(ref->w);
  } else {
    cudaFree(ref->yc);
    if (ref->w) cudaFree(ref->w);
  }
  delete ref;
  return WMD_OK;
}

WMD_EXPORT int wmd_set_wait_test(wmd_ctx* ctx, uint64_t wait_limit_ns, int withhold_first_stage) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  ctx->wait.limit_ns = wait_limit_ns ? wait_limit_ns : wmd::kWaitLimitNs;
  ctx->wait.withhold = withhold_first_stage ? 1 : 0;
  ctx->pw.wait = ctx->wait;
  return WMD_OK;
}

static int frames_common(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                         const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int align, wmd::FrameOutputs o_user,
                         bool outputs_host, cudaStream_t s) {
  const Mem cm = classify(coords);
  const uint32_t* dsel = nullptr;
  int rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s);
  if (rc) return rc;
  LaneScope lane_scope{ctx};
  if ((rc = lanes_prepare(ctx, sel, dsel, n_sel, stride, ref, s))) return rc;
  if (n_sel == 0) {
    // the reference returns 0.0 for every frame (plan.rs:1166-1168)
    if (o_user.rmsd) {
      if (outputs_host) std::fill(o_user.rmsd, o_user.rmsd + n_frames, 0.0);
      else CU(cudaMemsetAsync(o_user.rmsd, 0, (size_t)n_frames * sizeof(double), s), "memset");
    }
    return WMD_OK;
  }
  // outputs staged through device memory when the caller's are host memory
  wmd::FrameOutputs o = o_user;
  size_t off_rmsd = 0, off_cov = 0, off_x2 = 0, off_y2 = 0, total = 0;
  if (outputs_host) {
    auto take = [&](size_t bytes) { size_t at = total; total += (bytes + 255) & ~size_t(255); return at; };
    if (o_user.rmsd) off_rmsd = take((size_t)n_frames * sizeof(double));
    if (o_user.cov) off_cov = take((size_t)n_frames * 9 * sizeof(float));
    if (o_user.sum_x2) off_x2 = take((size_t)n_frames * sizeof(float));
    if (o_user.sum_y2) off_y2 = take((size_t)n_frames * sizeof(float));
    rc = ensure(ctx, ctx->out_tmp, total);
    if (rc) return rc;
    char* base = static_cast<char*>(ctx->out_tmp.ptr);
    o.rmsd = o_user.rmsd ? reinterpret_cast<double*>(base + off_rmsd) : nullptr;
    o.cov = o_user.cov ? reinterpret_cast<float*>(base + off_cov) : nullptr;
    o.sum_x2 = o_user.sum_x2 ? reinterpret_cast<float*>(base + off_x2) : nullptr;
    o.sum_y2 = o_user.sum_y2 ? reinterpret_cast<float*>(base + off_y2) : nullptr;
  }
  if (is_host(cm)) rc = forward_host(ctx, coords, cm, n_frames, n_atoms, stride, dsel, ref, align, o, s);
  else rc = forward_device(ctx, coords, n_frames, n_atoms, stride, dsel, ref, align, o, s);
  if (rc) return rc;
  if (outputs_host) {
    if (o.rmsd) CU(cudaMemcpyAsync(o_user.rmsd, o.rmsd, (size_t)n_frames * 8, cudaMemcpyDeviceToHost, s), "D2H");
    if (o.cov) CU(cudaMemcpyAsync(o_user.cov, o.cov, (size_t)n_frames * 36, cudaMemcpyDeviceToHost, s), "D2H");
    if (o.sum_x2) CU(cudaMemcpyAsync(o_user.sum_x2, o.sum_x2, (size_t)n_frames * 4, cudaMemcpyDeviceToHost, s), "D2H");
    if (o.sum_y2) CU(cudaMemcpyAsync(o_user.sum_y2, o.sum_y2, (size_t)n_frames * 4, cudaMemcpyDeviceToHost, s), "D2H");
  }
  if (outputs_host || is_host(cm) || (sel && classify(sel) != Mem::Device)) {
    CU(cudaStreamSynchronize(s), "synchronize");
    return check_status(ctx);
  }
  return WMD_OK;
}

WMD_EXPORT int wmd_rmsd_frames(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                               const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int align, double* out,
                               void* stream) {
  int rc = check_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref);
  if (rc) return rc;
  if (n_frames > 0 && !out) return set_err(ctx, WMD_ERR_INVALID_ARG, "out is null");
  DeviceGuard g(ctx->device);
  if ((rc = check_status(ctx))) return rc;
  if (n_frames == 0) return WMD_OK;
  wmd::FrameOutputs o;
  o.rmsd = out;
  return frames_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, align, o, is_host(classify(out)),
                       static_cast<cudaStream_t>(stream));
}

WMD_EXPORT int wmd_rmsd_covariance(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                   const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, float* cov, float* sum_x2,
                                   float* sum_y2, void* stream) {
  int rc = check_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref);
  if (rc) return rc;
  if (n_frames > 0 && (!cov || !sum_x2 || !sum_y2)) return set_err(ctx, WMD_ERR_INVALID_ARG, "output is null");
  DeviceGuard g(ctx->device);
  if ((rc = check_status(ctx))) return rc;
  if (n_frames == 0) return WMD_OK;
  const bool oh = is_host(classify(cov));
  if (oh != is_host(classify(sum_x2)) || oh != is_host(classify(sum_y2)))
    return set_err(ctx, WMD_ERR_INVALID_ARG, "cov, sum_x2 and sum_y2 must all be host or all be device memory");
  if (n_sel == 0) {
    // covariance of an empty selection is zero
    if (oh) {
      std::fill(cov, cov + n_frames * 9, 0.f);
      std::fill(sum_x2, sum_x2 + n_frames, 0.f);
      std::fill(sum_y2, sum_y2 + n_frames, 0.f);
      return WMD_OK;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CU(cudaMemsetAsync(cov, 0, (size_t)n_frames * 36, s), "memset");
    CU(cudaMemsetAsync(sum_x2, 0, (size_t)n_frames * 4, s), "memset");
    CU(cudaMemsetAsync(sum_y2, 0, (size_t)n_frames * 4, s), "memset");
    return WMD_OK;
  }
  wmd::FrameOutputs o;
  o.cov = cov;
  o.sum_x2 = sum_x2;
  o.sum_y2 = sum_y2;
  return frames_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, 1, o, oh,
                       static_cast<cudaStream_t>(stream));
}

static int require_device(wmd_ctx* ctx, const void* p, const char* name) {
  if (p && classify(p) != Mem::Device)
    return set_err(ctx, WMD_ERR_INVALID_ARG, "%s must be device memory for this entry point", name);
  return WMD_OK;
}

// ---------------------------------------------------------------------------
// superposition (AlignPlan / RotationMatrixPlan / SuperposePlan)
// ---------------------------------------------------------------------------

// Device-resident frames: statistics, per-frame transforms into dxf32 (if not
// null) and, when dout is not null, every atom moved into dout.
// Per-group RMSD run after the transforms of each batch (RmsdPerResPlan).
struct GroupJob {
  const uint32_t* goff = nullptr;
  const uint32_t* gatoms = nullptr;
  const uint32_t* blocks = nullptr;
  int64_t n_blocks = 0;
  int64_t contig_base = -1;
  int64_t n_groups = 0;
  const float* ref_all = nullptr;
  float* out = nullptr;  // [n_frames of this call][n_groups], device
};

static int superpose_device(wmd_ctx* ctx, const float* dcoords, int64_t n_frames, int64_t n_atoms, int stride,
                            const uint32_t* dsel, const wmd_ref* ref, int norotate, float* dxf32, float* dout,
                            cudaStream_t s, const GroupJob* grp = nullptr, double* xf64_out = nullptr) {
  if (n_frames == 0) return WMD_OK;
  wmd::FrameLaunch L = base_launch(ctx, ref, n_atoms, stride, dsel);
  L.align = 1;
  L.gather = dsel != nullptr || (reinterpret_cast<uintptr_t>(dcoords) & 15u) != 0;
  L.coords = dcoords;
  L.n_frames = n_frames;
  apply_lanes(ctx, L, dsel);
  wmd::frame_plan(L, ctx->sm_count);
  const int tiles = wmd::frame_tiles(L);
  const size_t per_frame = (size_t)std::max(tiles, 1) * wmd::kStatDoubles * sizeof(double);
  const int64_t batch = frame_batch(kPartialBytesMax / per_frame, n_frames);
  int rc;
  if ((rc = ensure(ctx, ctx->partial, per_frame * (size_t)batch)) ||
      (rc = ensure(ctx, ctx->rot, (size_t)batch * wmd::kStatDoubles * sizeof(double))))
    return rc;
  for (int64_t f0 = 0; f0 < n_frames; f0 += batch) {
    const int64_t nf = std::min(batch, n_frames - f0);
    wmd::FrameLaunch B = L;
    B.coords = dcoords + (size_t)f0 * n_atoms * stride;
    keep_aligned(B);
    B.n_frames = nf;
    B.partial = static_cast<double*>(ctx->partial.ptr);
    B.grid = wmd::frame_grid(B, ctx->sm_count, false);
    if (ref->info.n_sel > 0) {
      if (ref->info.w) CU(wmd::launch_rmsd_stream_weighted(B, s), "superpose statistics");
      else CU(wmd::launch_rmsd_stream(B, s), "superpose statistics");
    }
    double* xf = static_cast<double*>(ctx->rot.ptr);
    CU(wmd::launch_superpose_finalize(B, norotate, xf, dxf32 ? dxf32 + f0 * 12 : nullptr, s), "superpose transforms");
    if (xf64_out)
      CU(cudaMemcpyAsync(xf64_out + f0 * wmd::kStatDoubles, xf, (size_t)nf * wmd::kStatDoubles * sizeof(double),
                         cudaMemcpyDeviceToDevice, s),
         "copy transforms");
    if (dout)
      CU(wmd::launch_superpose_apply(B.coords, nf, n_atoms, stride, xf, dout + (size_t)f0 * n_atoms * 3, ctx->sm_count,
                                     ctx->status_dev, s),
         "superpose apply");
    if (grp)
      CU(wmd::launch_group_rmsd(B.coords, nf, n_atoms, stride, xf, grp->goff, grp->gatoms, grp->contig_base,
                                grp->blocks, grp->n_blocks, grp->n_groups, grp->ref_all,
                                grp->out + f0 * grp->n_groups, ctx->sm_count, s),
         "per-group rmsd");
  }
  return WMD_OK;
}

// Calls fn(device_frames, f0, nf) for consecutive runs of frames: in place for
// device memory; for host memory through the context's two chunk buffers, the
// H2D copy of the next chunk overlapping the work on this one.
template <class Fn>
static int for_each_chunk(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                          cudaStream_t s, Fn fn) {
  const Mem cm = classify(coords);
  if (cm == Mem::Device) return fn(coords, (int64_t)0, n_frames);
  const size_t frame_bytes = (size_t)n_atoms * stride * sizeof(float);
  const int64_t chunk = std::max<int64_t>(
      1, std::min<int64_t>(n_frames, (int64_t)(kChunkBytes / std::max<size_t>(frame_bytes, 1))));
  int rc;
  for (int b = 0; b < 2; ++b) {
    if ((rc = ensure(ctx, ctx->chunk[b], (size_t)chunk * frame_bytes + 16))) return rc;
    if (cm == Mem::PageableHost && (rc = ensure_host(ctx, ctx->stage[b], (size_t)chunk * frame_bytes + 16))) return rc;
  }
  CU(cudaEventRecord(ctx->kern_done[0], s), "event");
  CU(cudaEventRecord(ctx->kern_done[1], s), "event");
  CU(cudaEventRecord(ctx->h2d_done[0], ctx->copy_stream), "event");
  CU(cudaEventRecord(ctx->h2d_done[1], ctx->copy_stream), "event");
  int64_t k = 0;
  for (int64_t f0 = 0; f0 < n_frames; f0 += chunk, ++k) {
    const int b = (int)(k & 1);
    const int64_t nf = std::min(chunk, n_frames - f0);
    const size_t bytes = (size_t)nf * frame_bytes;
    const char* src = reinterpret_cast<const char*>(coords) + (size_t)f0 * frame_bytes;
    if (cm == Mem::PageableHost) {
      CU(cudaEventSynchronize(ctx->h2d_done[b]), "staging wait");
      std::memcpy(ctx->stage[b].ptr, src, bytes);
      src = static_cast<const char*>(ctx->stage[b].ptr);
    }
    CU(cudaStreamWaitEvent(ctx->copy_stream, ctx->kern_done[b], 0), "stream wait");
    CU(cudaMemcpyAsync(ctx->chunk[b].ptr, src, bytes, cudaMemcpyHostToDevice, ctx->copy_stream), "H2D");
    CU(cudaEventRecord(ctx->h2d_done[b], ctx->copy_stream), "event");
    CU(cudaStreamWaitEvent(s, ctx->h2d_done[b], 0), "stream wait");
    if ((rc = fn(static_cast<const float*>(ctx->chunk[b].ptr), f0, nf))) return rc;
    CU(cudaEventRecord(ctx->kern_done[b], s), "event");
  }
  return WMD_OK;
}


static int superpose_common(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                            const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int norotate, float* out,
                            float* transforms, cudaStream_t s) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!ref) return set_err(ctx, WMD_ERR_INVALID_ARG, "reference is null");
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_frames > 0 && !coords) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords is null");
  if (n_sel != ref->info.n_sel)
    return set_err(ctx, WMD_ERR_MISMATCH, "reference has %lld atoms but the selection has %lld",
                   (long long)ref->info.n_sel, (long long)n_sel);
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if (n_frames == 0) return WMD_OK;
  const uint32_t* dsel = nullptr;
  if ((rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s))) return rc;
  LaneScope lane_scope{ctx};
  if ((rc = lanes_prepare(ctx, sel, dsel, n_sel, stride, ref, s))) return rc;
  const Mem cm = classify(coords);
  const bool out_host = out && is_host(classify(out));
  const bool xf_host = transforms && is_host(classify(transforms));
  if (cm == Mem::Device && !out_host && !xf_host)
    return superpose_device(ctx, coords, n_frames, n_atoms, stride, dsel, ref, norotate, transforms, out, s);
  // host memory somewhere: chunks of frames through device buffers
  const size_t frame_bytes = (size_t)n_atoms * stride * sizeof(float);
  const size_t out_frame_bytes = (size_t)n_atoms * 3 * sizeof(float);
  const int64_t chunk = std::max<int64_t>(
      1, std::min<int64_t>(n_frames, (int64_t)(kChunkBytes / std::max<size_t>(frame_bytes, 1))));
  if (cm != Mem::Device) {
    for (int b = 0; b < 2; ++b) {
      if ((rc = ensure(ctx, ctx->chunk[b], (size_t)chunk * frame_bytes + 16))) return rc;
      if (cm == Mem::PageableHost && (rc = ensure_host(ctx, ctx->stage[b], (size_t)chunk * frame_bytes + 16))) return rc;
    }
    CU(cudaEventRecord(ctx->kern_done[0], s), "event");
    CU(cudaEventRecord(ctx->kern_done[1], s), "event");
    CU(cudaEventRecord(ctx->h2d_done[0], ctx->copy_stream), "event");
    CU(cudaEventRecord(ctx->h2d_done[1], ctx->copy_stream), "event");
  }
  if (out_host && (rc = ensure(ctx, ctx->out_chunk, (size_t)chunk * out_frame_bytes + 16))) return rc;
  if (xf_host && (rc = ensure(ctx, ctx->out_tmp, (size_t)chunk * 12 * sizeof(float)))) return rc;
  int64_t k = 0;
  for (int64_t f0 = 0; f0 < n_frames; f0 += chunk, ++k) {
    const int b = (int)(k & 1);
    const int64_t nf = std::min(chunk, n_frames - f0);
    const float* dc = coords + (size_t)f0 * n_atoms * stride;
    if (cm != Mem::Device) {
      const size_t bytes = (size_t)nf * frame_bytes;
      const char* src = reinterpret_cast<const char*>(dc);
      if (cm == Mem::PageableHost) {
        CU(cudaEventSynchronize(ctx->h2d_done[b]), "staging wait");
        std::memcpy(ctx->stage[b].ptr, src, bytes);
        src = static_cast<const char*>(ctx->stage[b].ptr);
      }
      CU(cudaStreamWaitEvent(ctx->copy_stream, ctx->kern_done[b], 0), "stream wait");
      CU(cudaMemcpyAsync(ctx->chunk[b].ptr, src, bytes, cudaMemcpyHostToDevice, ctx->copy_stream), "H2D");
      CU(cudaEventRecord(ctx->h2d_done[b], ctx->copy_stream), "event");
      CU(cudaStreamWaitEvent(s, ctx->h2d_done[b], 0), "stream wait");
      dc = static_cast<const float*>(ctx->chunk[b].ptr);
    }
    float* dout = !out ? nullptr : out_host ? static_cast<float*>(ctx->out_chunk.ptr) : out + (size_t)f0 * n_atoms * 3;
    float* dxf = !transforms ? nullptr : xf_host ? static_cast<float*>(ctx->out_tmp.ptr) : transforms + f0 * 12;
    if ((rc = superpose_device(ctx, dc, nf, n_atoms, stride, dsel, ref, norotate, dxf, dout, s))) return rc;
    if (cm != Mem::Device) CU(cudaEventRecord(ctx->kern_done[b], s), "event");
    if (out_host)
      CU(cudaMemcpyAsync(out + (size_t)f0 * n_atoms * 3, dout, (size_t)nf * out_frame_bytes, cudaMemcpyDeviceToHost, s),
         "D2H");
    if (xf_host)
      CU(cudaMemcpyAsync(transforms + f0 * 12, dxf, (size_t)nf * 12 * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
  }
  CU(cudaStreamSynchronize(s), "synchronize");
  return check_status(ctx);
}

WMD_EXPORT int wmd_superpose_transforms(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms,
                                        int stride, const uint32_t* sel, int64_t n_sel, const wmd_ref* ref,
                                        int norotate, float* transforms, void* stream) {
  if (ctx && n_frames > 0 && !transforms) return set_err(ctx, WMD_ERR_INVALID_ARG, "transforms is null");
  return superpose_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, norotate, nullptr, transforms,
                          static_cast<cudaStream_t>(stream));
}

WMD_EXPORT int wmd_superpose(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                             const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, int norotate, float* out,
                             float* transforms, void* stream) {
  if (ctx && n_frames > 0 && !out) return set_err(ctx, WMD_ERR_INVALID_ARG, "out is null");
  return superpose_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, norotate, out, transforms,
                          static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// fluctuations (RmsfPlan / AtomicFluctPlan / BfactorsPlan / AtomicAdpPlan) and
// per-group RMSD (RmsdPerResPlan)
// ---------------------------------------------------------------------------

WMD_EXPORT int wmd_rmsf(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                        const uint32_t* sel, int64_t n_sel, float* rmsf, float* adp, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_frames > 0 && n_sel > 0 && !coords) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords is null");
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  if (n_sel > 0 && !rmsf && !adp) return set_err(ctx, WMD_ERR_INVALID_ARG, "rmsf and adp are both null");
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_sel == 0) return WMD_OK;
  const bool rh = rmsf && is_host(classify(rmsf)), ah = adp && is_host(classify(adp));
  if (n_frames == 0) {
    // no frames: RMSF 0 (rms.rs:194-196); the ADP tensor has no rows then
    if (rmsf) {
      if (rh) std::fill(rmsf, rmsf + n_sel, 0.f);
      else CU(cudaMemsetAsync(rmsf, 0, (size_t)n_sel * sizeof(float), s), "memset");
    }
    return WMD_OK;
  }
  const uint32_t* dsel = nullptr;
  if ((rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s))) return rc;
  const int G = wmd::fluct_groups(n_sel, n_frames, ctx->sm_count);
  const size_t mom = (size_t)n_sel * wmd::kFluctMoments * sizeof(double);
  if ((rc = ensure(ctx, ctx->fl_part, mom * (size_t)G)) || (rc = ensure(ctx, ctx->fl_acc, mom)) ||
      (rc = ensure(ctx, ctx->fl_shift, (size_t)n_sel * 3 * sizeof(float))))
    return rc;
  double* acc = static_cast<double*>(ctx->fl_acc.ptr);
  CU(cudaMemsetAsync(acc, 0, mom, s), "memset");
  rc = for_each_chunk(ctx, coords, n_frames, n_atoms, stride, s, [&](const float* dc, int64_t f0, int64_t nf) -> int {
    if (f0 == 0)
      CU(wmd::launch_fluct_shift(dc, n_atoms, stride, dsel, n_sel, static_cast<float*>(ctx->fl_shift.ptr),
                                 ctx->status_dev, s),
         "fluctuation shift");
    const int Gc = wmd::fluct_groups(n_sel, nf, ctx->sm_count);
    CU(wmd::launch_fluct_chunk(dc, nf, n_atoms, stride, dsel, n_sel, static_cast<const float*>(ctx->fl_shift.ptr),
                               std::min(Gc, G), static_cast<double*>(ctx->fl_part.ptr), acc, s),
       "fluctuation moments");
    return WMD_OK;
  });
  if (rc) return rc;
  float* drmsf = rmsf;
  float* dadp = adp;
  if (rh || ah) {
    if ((rc = ensure(ctx, ctx->out_tmp, (size_t)n_sel * 7 * sizeof(float)))) return rc;
    float* tmp = static_cast<float*>(ctx->out_tmp.ptr);
    if (rh) drmsf = tmp;
    if (ah) dadp = tmp + n_sel;
  }
  CU(wmd::launch_fluct_finalize(acc, n_sel, n_frames, drmsf, dadp, s), "fluctuation finalize");
  if (rh) CU(cudaMemcpyAsync(rmsf, drmsf, (size_t)n_sel * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
  if (ah) CU(cudaMemcpyAsync(adp, dadp, (size_t)n_sel * 6 * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
  if (rh || ah || is_host(classify(coords))) {
    CU(cudaStreamSynchronize(s), "synchronize");
    return check_status(ctx);
  }
  return WMD_OK;
}

WMD_EXPORT int wmd_group_ref_upload(wmd_ctx* ctx, const float* ref_all, int64_t n_atoms, int stride,
                                    const uint32_t* group_offsets, const uint32_t* group_atoms, int64_t n_groups,
                                    wmd_group_ref** out) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!out) return set_err(ctx, WMD_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_atoms < 0 || n_groups < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_groups > 0 && (!group_offsets || !group_atoms || (n_atoms > 0 && !ref_all)))
    return set_err(ctx, WMD_ERR_INVALID_ARG, "ref_all, group_offsets and group_atoms are required");
  DeviceGuard g(ctx->device);
  // host copies of everything, validated here once so the kernels read no
  // index out of range
  std::vector<uint32_t> off((size_t)n_groups + 1, 0), atoms;
  std::vector<float> ref((size_t)n_atoms * 3);
  if (n_groups > 0) {
    if (classify(group_offsets) == Mem::Device)
      CU(cudaMemcpy(off.data(), group_offsets, off.size() * 4, cudaMemcpyDeviceToHost), "download");
    else
      std::memcpy(off.data(), group_offsets, off.size() * 4);
    if (off[0] != 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "group_offsets[0] must be 0");
    for (int64_t gi = 0; gi < n_groups; ++gi)
      if (off[gi + 1] < off[gi]) return set_err(ctx, WMD_ERR_INVALID_ARG, "group_offsets must not decrease");
    atoms.resize(off[n_groups]);
    if (!atoms.empty()) {
      if (classify(group_atoms) == Mem::Device)
        CU(cudaMemcpy(atoms.data(), group_atoms, atoms.size() * 4, cudaMemcpyDeviceToHost), "download");
      else
        std::memcpy(atoms.data(), group_atoms, atoms.size() * 4);
    }
    for (uint32_t a : atoms)
      if ((int64_t)a >= n_atoms)
        return set_err(ctx, WMD_ERR_INVALID_ARG, "group atom index %u out of range for %lld atoms", a,
                       (long long)n_atoms);
  }
  if (n_atoms > 0 && ref_all) {
    std::vector<float> raw((size_t)n_atoms * stride);
    if (classify(ref_all) == Mem::Device)
      CU(cudaMemcpy(raw.data(), ref_all, raw.size() * 4, cudaMemcpyDeviceToHost), "download");
    else
      std::memcpy(raw.data(), ref_all, raw.size() * 4);
    for (int64_t a = 0; a < n_atoms; ++a)
      for (int c = 0; c < 3; ++c) ref[a * 3 + c] = raw[a * stride + c];
  }
  std::vector<uint32_t> blocks((size_t)n_groups + 1, 0);
  const int nb = n_groups > 0 ? wmd::group_blocks(off.data(), n_groups, blocks.data()) : 0;
  wmd_group_ref* r = new wmd_group_ref();
  if (!atoms.empty()) {
    bool contig = true;
    for (size_t q = 0; q < atoms.size() && contig; ++q) contig = atoms[q] == atoms[0] + q;
    if (contig) r->contig_base = atoms[0];
  }
  r->n_atoms = n_atoms;
  r->n_groups = n_groups;
  r->n_blocks = nb;
  size_t total = 0;
  auto take = [&](size_t bytes) {
    const size_t at = total;
    total += (bytes + 255) & ~size_t(255);
    return at;
  };
  const size_t o_off = take(off.size() * 4), o_atoms = take(std::max<size_t>(atoms.size(), 1) * 4),
               o_blocks = take(((size_t)nb + 1) * 4), o_ref = take(std::max<size_t>(ref.size(), 1) * 4);
  cudaError_t e = cudaMalloc(&r->mem, total);
  if (e != cudaSuccess) {
    delete r;
    cudaGetLastError();
    return set_err(ctx, WMD_ERR_OOM, "cuda driver error: group allocation failed: %s", cudaGetErrorString(e));
  }
  char* base = static_cast<char*>(r->mem);
  r->goff = reinterpret_cast<uint32_t*>(base + o_off);
  r->gatoms = reinterpret_cast<uint32_t*>(base + o_atoms);
  r->blocks = reinterpret_cast<uint32_t*>(base + o_blocks);
  r->ref_all = reinterpret_cast<float*>(base + o_ref);
  e = cudaMemcpy(r->goff, off.data(), off.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !atoms.empty()) e = cudaMemcpy(r->gatoms, atoms.data(), atoms.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(r->blocks, blocks.data(), ((size_t)nb + 1) * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !ref.empty()) e = cudaMemcpy(r->ref_all, ref.data(), ref.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(r->mem);
    delete r;
    return cuda_err(ctx, e, "upload groups");
  }
  *out = r;
  return WMD_OK;
}

WMD_EXPORT int wmd_group_ref_free(wmd_ctx* ctx, wmd_group_ref* groups) {
  if (!groups) return WMD_OK;
  if (ctx) {
    DeviceGuard g(ctx->device);
    cudaFree(groups->mem);
  } else {
    cudaFree(groups->mem);
  }
  delete groups;
  return WMD_OK;
}

WMD_EXPORT int wmd_rmsd_per_group(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                  const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const wmd_group_ref* groups,
                                  int align, float* out, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (!groups) return set_err(ctx, WMD_ERR_INVALID_ARG, "groups is null");
  if (groups->n_atoms != n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "groups were made for %lld atoms but frames have %lld",
                   (long long)groups->n_atoms, (long long)n_atoms);
  if (n_frames > 0 && !coords) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords is null");
  if (n_frames > 0 && groups->n_groups > 0 && !out) return set_err(ctx, WMD_ERR_INVALID_ARG, "out is null");
  if (align && !ref) return set_err(ctx, WMD_ERR_INVALID_ARG, "reference is null");
  if (align && ref->info.w)
    return set_err(ctx, WMD_ERR_INVALID_ARG, "per-group RMSD superposes without weights; pass an unweighted reference");
  if (align && n_sel != ref->info.n_sel)
    return set_err(ctx, WMD_ERR_MISMATCH, "reference has %lld atoms but the selection has %lld",
                   (long long)ref->info.n_sel, (long long)n_sel);
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  const int64_t n_groups = groups->n_groups;
  if (n_frames == 0 || n_groups == 0) return WMD_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t* dsel = nullptr;
  if (align && (rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s))) return rc;
  LaneScope lane_scope{ctx};
  if (align && (rc = lanes_prepare(ctx, sel, dsel, n_sel, stride, ref, s))) return rc;
  GroupJob job;
  job.goff = groups->goff;
  job.gatoms = groups->gatoms;
  job.blocks = groups->blocks;
  job.n_blocks = groups->n_blocks;
  job.contig_base = groups->contig_base;
  job.n_groups = n_groups;
  job.ref_all = groups->ref_all;
  const bool oh = is_host(classify(out));
  const size_t row = (size_t)n_groups * sizeof(float);
  rc = for_each_chunk(ctx, coords, n_frames, n_atoms, stride, s, [&](const float* dc, int64_t f0, int64_t nf) -> int {
    GroupJob jb = job;
    if (oh) {
      int r2 = ensure(ctx, ctx->out_chunk, (size_t)nf * row);
      if (r2) return r2;
      jb.out = static_cast<float*>(ctx->out_chunk.ptr);
    } else {
      jb.out = out + f0 * n_groups;
    }
    if (align) {
      int r2 = superpose_device(ctx, dc, nf, n_atoms, stride, dsel, ref, 0, nullptr, nullptr, s, &jb);
      if (r2) return r2;
    } else {
      CU(wmd::launch_group_rmsd(dc, nf, n_atoms, stride, nullptr, jb.goff, jb.gatoms, jb.contig_base, jb.blocks,
                                jb.n_blocks, n_groups, jb.ref_all, jb.out, ctx->sm_count, s),
         "per-group rmsd");
    }
    if (oh) CU(cudaMemcpyAsync(out + f0 * n_groups, jb.out, (size_t)nf * row, cudaMemcpyDeviceToHost, s), "D2H");
    return WMD_OK;
  });
  if (rc) return rc;
  if (oh || is_host(classify(coords))) {
    CU(cudaStreamSynchronize(s), "synchronize");
    return check_status(ctx);
  }
  return WMD_OK;
}

WMD_EXPORT int wmd_rmsd_forward(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, double* out, double* stats,
                                void* stream) {
  int rc = check_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref);
  if (rc) return rc;
  DeviceGuard g(ctx->device);
  if ((rc = check_status(ctx))) return rc;
  if (n_frames == 0) return WMD_OK;
  if ((rc = require_device(ctx, coords, "coords")) || (rc = require_device(ctx, sel, "sel")) ||
      (rc = require_device(ctx, out, "out")) || (rc = require_device(ctx, stats, "stats")))
    return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_sel == 0) {
    if (out) CU(cudaMemsetAsync(out, 0, (size_t)n_frames * 8, s), "memset");
    if (stats) CU(cudaMemsetAsync(stats, 0, (size_t)n_frames * wmd::kStatDoubles * 8, s), "memset");
    return WMD_OK;
  }
  if (!sel && wmd::vg_usable(coords, nullptr, n_frames, n_atoms, stride, ctx->sm_count)) {
    wmd::VgLaunch V = vg_launch(ctx, ref, coords, n_frames, n_atoms);
    V.rmsd = out;
    V.stats = stats;
    {
      const char* why = "";
      const cudaError_t e = wmd::launch_vg(wmd::kVgFwd, V, ctx->sm_count, s, &why);
      if (e != cudaSuccess) return set_err(ctx, WMD_ERR_CUDA, "cuda driver error: rmsd forward (%s): %s", why, cudaGetErrorString(e));
    }
    return WMD_OK;
  }
  wmd::FrameOutputs o;
  o.rmsd = out;
  o.stats = stats;
  return forward_device(ctx, coords, n_frames, n_atoms, stride, sel, ref, 1, o, s);
}

// Gradient from the forward's records; per-frame weights as float (gf) or
// double with a stride (gd), or all 1.
static int backward_common(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                           const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const double* stats,
                           const float* gf, const double* gd, int64_t gstride, float* grad, cudaStream_t s) {
  if (!sel && wmd::vg_usable(coords, grad, n_frames, n_atoms, stride, ctx->sm_count)) {
    wmd::VgLaunch V = vg_launch(ctx, ref, coords, n_frames, n_atoms);
    V.stats = const_cast<double*>(stats);
    V.w = gd ? static_cast<const void*>(gd) : static_cast<const void*>(gf);
    V.w_f64 = gd != nullptr;
    V.w_stride = gd ? gstride : 1;
    V.grad = grad;
    {
      const char* why = "";
      const cudaError_t e = wmd::launch_vg(wmd::kVgBwd, V, ctx->sm_count, s, &why);
      if (e != cudaSuccess) return set_err(ctx, WMD_ERR_CUDA, "cuda driver error: rmsd backward (%s): %s", why, cudaGetErrorString(e));
    }
    return WMD_OK;
  }
  int rc = ensure(ctx, ctx->rot, (size_t)n_frames * wmd::kStatDoubles * sizeof(double));
  if (rc) return rc;
  wmd::FrameLaunch L = base_launch(ctx, ref, n_atoms, stride, sel);
  L.coords = coords;
  L.n_frames = n_frames;
  L.gather = sel != nullptr || (reinterpret_cast<uintptr_t>(coords) & 15u) != 0;
  L.grad = grad;
  L.grid = wmd::frame_grid(L, ctx->sm_count, true);
  CU(wmd::launch_rmsd_backward(L, stats, gf, gd, gstride, static_cast<double*>(ctx->rot.ptr), s),
     "rmsd backward launch");
  return WMD_OK;
}

static int backward_checks(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                           const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const double* stats,
                           const void* weights, float* grad) {
  int rc = check_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref);
  if (rc) return rc;
  if (n_frames > 0 && n_sel > 0 && (!stats || !grad))
    return set_err(ctx, WMD_ERR_INVALID_ARG, "stats and grad are required");
  if ((rc = require_device(ctx, coords, "coords")) || (rc = require_device(ctx, sel, "sel")) ||
      (rc = require_device(ctx, stats, "stats")) || (rc = require_device(ctx, weights, "grad_rmsd")) ||
      (rc = require_device(ctx, grad, "grad")))
    return rc;
  return WMD_OK;
}

WMD_EXPORT int wmd_rmsd_backward(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                 const uint32_t* sel, int64_t n_sel, const wmd_ref* ref, const double* stats,
                                 const float* grad_rmsd, float* grad, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if ((rc = backward_checks(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, stats, grad_rmsd, grad)))
    return rc;
  if (n_frames == 0 || n_sel == 0) return WMD_OK;
  return backward_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, stats, grad_rmsd, nullptr, 0, grad,
                         static_cast<cudaStream_t>(stream));
}

WMD_EXPORT int wmd_rmsd_backward_f64(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms,
                                     int stride, const uint32_t* sel, int64_t n_sel, const wmd_ref* ref,
                                     const double* stats, const double* grad_rmsd, int64_t grad_stride, float* grad,
                                     void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (grad_stride < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "grad_stride must be >= 0");
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if ((rc = backward_checks(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, stats, grad_rmsd, grad)))
    return rc;
  if (n_frames == 0 || n_sel == 0) return WMD_OK;
  return backward_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, stats, nullptr, grad_rmsd,
                         grad_stride, grad, static_cast<cudaStream_t>(stream));
}

WMD_EXPORT int wmd_rmsd_value_and_grad(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms,
                                       int stride, const uint32_t* sel, int64_t n_sel, const wmd_ref* ref,
                                       const double* weights, int64_t weight_stride, double* rmsd, float* grad,
                                       void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (weight_stride < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "weight_stride must be >= 0");
  int rc = check_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref);
  if (rc) return rc;
  DeviceGuard g(ctx->device);
  if ((rc = check_status(ctx))) return rc;
  if (n_frames == 0) return WMD_OK;
  if (!grad) return set_err(ctx, WMD_ERR_INVALID_ARG, "grad is required");
  if ((rc = require_device(ctx, coords, "coords")) || (rc = require_device(ctx, sel, "sel")) ||
      (rc = require_device(ctx, weights, "weights")) || (rc = require_device(ctx, rmsd, "rmsd")) ||
      (rc = require_device(ctx, grad, "grad")))
    return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n_sel == 0) {
    if (rmsd) CU(cudaMemsetAsync(rmsd, 0, (size_t)n_frames * 8, s), "memset");
    return WMD_OK;
  }
  if (!sel && wmd::vg_usable(coords, grad, n_frames, n_atoms, stride, ctx->sm_count)) {
    wmd::VgLaunch V = vg_launch(ctx, ref, coords, n_frames, n_atoms);
    V.rmsd = rmsd;
    V.w = weights;
    V.w_f64 = 1;
    V.w_stride = weight_stride;
    V.grad = grad;
    {
      const char* why = "";
      const cudaError_t e = wmd::launch_vg(wmd::kVgBoth, V, ctx->sm_count, s, &why);
      if (e != cudaSuccess) return set_err(ctx, WMD_ERR_CUDA, "cuda driver error: rmsd value and gradient (%s): %s", why, cudaGetErrorString(e));
    }
    return WMD_OK;
  }
  // any other shape: the forward into context scratch, then the backward
  if ((rc = ensure(ctx, ctx->vg_stats, (size_t)n_frames * wmd::kStatDoubles * sizeof(double)))) return rc;
  double* st = static_cast<double*>(ctx->vg_stats.ptr);
  wmd::FrameOutputs o;
  o.rmsd = rmsd;
  o.stats = st;
  if ((rc = forward_device(ctx, coords, n_frames, n_atoms, stride, sel, ref, 1, o, s))) return rc;
  return backward_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, ref, st, nullptr, weights,
                         weights ? weight_stride : 0, grad, s);
}

static int pairwise_common(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                           const uint32_t* sel, int64_t n_sel, int metric, int mode, int part, int parts, float* out,
                           void* stream);

WMD_EXPORT int wmd_pairwise_rmsd(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                 const uint32_t* sel, int64_t n_sel, int metric, int mode, float* out, void* stream) {
  return pairwise_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, metric, mode, 0, 1, out, stream);
}

WMD_EXPORT int wmd_pairwise_rmsd_part(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms,
                                      int stride, const uint32_t* sel, int64_t n_sel, int metric, int mode, int part,
                                      int parts, float* out, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (parts < 1 || part < 0 || part >= parts)
    return set_err(ctx, WMD_ERR_INVALID_ARG, "part %d of %d: need 0 <= part < parts", part, parts);
  if (metric == WMD_PAIR_DME && parts > 1)
    return set_err(ctx, WMD_ERR_UNSUPPORTED, "the dme metric is not partitioned (call with parts = 1)");
  return pairwise_common(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, metric, mode, part, parts, out, stream);
}

static int pairwise_common(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                           const uint32_t* sel, int64_t n_sel, int metric, int mode, int part, int parts, float* out,
                           void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (metric == WMD_PAIR_DME) return wmd_pairwise_dme(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, nullptr, out, stream);
  if (metric != WMD_PAIR_RMS && metric != WMD_PAIR_NOFIT)
    return set_err(ctx, WMD_ERR_UNSUPPORTED, "pairwise metric %d is not provided (rms=0, nofit=1, dme=2)", metric);
  if (mode < WMD_MODE_FP32 || mode > WMD_MODE_FP64)
    return set_err(ctx, WMD_ERR_INVALID_ARG, "unknown pairwise mode %d", mode);
  if (n_frames > 0 && (!coords || !out)) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords/out is null");
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if (n_frames == 0) return WMD_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Mem cm = classify(coords), om = classify(out);
  const uint32_t* dsel = nullptr;
  if ((rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s))) return rc;
  const float* dcoords = coords;
  if (is_host(cm)) {
    const size_t bytes = (size_t)n_frames * n_atoms * stride * sizeof(float);
    if ((rc = ensure(ctx, ctx->aux, bytes))) return rc;
    CU(cudaMemcpyAsync(ctx->aux.ptr, coords, bytes, cudaMemcpyHostToDevice, s), "H2D");
    dcoords = static_cast<const float*>(ctx->aux.ptr);
  }
  float* dout = out;
  const size_t out_bytes = (size_t)n_frames * n_frames * sizeof(float);
  if (is_host(om)) {
    if ((rc = ensure(ctx, ctx->out_tmp, out_bytes))) return rc;
    dout = static_cast<float*>(ctx->out_tmp.ptr);
  }
  std::string msg;
  ctx->pw.part = part;
  ctx->pw.parts = parts;
  const int prc = wmd::pairwise_run(ctx->pw, ctx->sm_count, dcoords, n_frames, n_atoms, stride, dsel, n_sel, metric,
                                    mode, dout, ctx->status_dev, s, &msg);
  ctx->pw.part = 0;
  ctx->pw.parts = 1;
  if (prc) return set_err(ctx, prc, "%s", msg.c_str());
  if (is_host(om)) CU(cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, s), "D2H");
  if (is_host(om) || is_host(cm) || (sel && classify(sel) != Mem::Device)) {
    CU(cudaStreamSynchronize(s), "synchronize");
    return check_status(ctx);
  }
  return WMD_OK;
}

WMD_EXPORT int wmd_pairwise_dme(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                const uint32_t* sel, int64_t n_sel, const float* box, float* out, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_frames > 0 && (!coords || !out)) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords/out is null");
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  if ((n_frames + 31) / 32 > 65535) return set_err(ctx, WMD_ERR_UNSUPPORTED, "too many frames for one pairwise call");
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if (n_frames == 0) return WMD_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Mem cm = classify(coords), om = classify(out), bm = box ? classify(box) : Mem::Device;
  const uint32_t* dsel = nullptr;
  if ((rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s))) return rc;
  // host inputs: coordinates, then the box lengths, in the context's staging buffer
  const size_t cbytes = is_host(cm) ? ((size_t)n_frames * n_atoms * stride * sizeof(float) + 255) / 256 * 256 : 0;
  const size_t bbytes = box && is_host(bm) ? (size_t)n_frames * 3 * sizeof(float) : 0;
  if (cbytes + bbytes && (rc = ensure(ctx, ctx->aux, cbytes + bbytes))) return rc;
  const float* dcoords = coords;
  if (cbytes) {
    CU(cudaMemcpyAsync(ctx->aux.ptr, coords, (size_t)n_frames * n_atoms * stride * sizeof(float),
                       cudaMemcpyHostToDevice, s),
       "H2D");
    dcoords = static_cast<const float*>(ctx->aux.ptr);
  }
  const float* dbox = box;
  if (bbytes) {
    float* bd = reinterpret_cast<float*>(static_cast<char*>(ctx->aux.ptr) + cbytes);
    CU(cudaMemcpyAsync(bd, box, bbytes, cudaMemcpyHostToDevice, s), "H2D");
    dbox = bd;
  }
  float* dout = out;
  const size_t out_bytes = (size_t)n_frames * n_frames * sizeof(float);
  if (is_host(om)) {
    if ((rc = ensure(ctx, ctx->out_tmp, out_bytes))) return rc;
    dout = static_cast<float*>(ctx->out_tmp.ptr);
  }
  CU(wmd::launch_pair_dme(dcoords, n_frames, n_atoms, stride, dsel, n_sel, dbox, dout, ctx->status_dev, s),
     "pairwise dme");
  if (is_host(om)) CU(cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, s), "D2H");
  if (is_host(om) || is_host(cm) || bbytes || (sel && classify(sel) != Mem::Device)) {
    CU(cudaStreamSynchronize(s), "synchronize");
    return check_status(ctx);
  }
  return WMD_OK;
}

WMD_EXPORT int wmd_cluster_dbscan(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                  const uint32_t* sel, int64_t n_sel, int mode, float eps, int64_t min_samples,
                                  int32_t* labels, uint32_t* centroids, uint32_t* sizes, int64_t* n_clusters,
                                  void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!n_clusters) return set_err(ctx, WMD_ERR_INVALID_ARG, "n_clusters is null");
  *n_clusters = 0;
  if (!(eps > 0.0f)) return set_err(ctx, WMD_ERR_INVALID_ARG, "parse error: trajectory_cluster DBSCAN eps must be > 0");
  if (n_sel == 0) return set_err(ctx, WMD_ERR_MISMATCH, "mismatch: trajectory_cluster requires a non-empty selection");
  if (n_frames < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_frames > (int64_t)0x7fffffff) return set_err(ctx, WMD_ERR_UNSUPPORTED, "too many frames for clustering");
  if (n_frames > 0 && (!labels || !centroids || !sizes))
    return set_err(ctx, WMD_ERR_INVALID_ARG, "labels, centroids and sizes are required");
  if (n_frames == 0) return WMD_OK;
  DeviceGuard g(ctx->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  const size_t mat = (size_t)n_frames * n_frames * sizeof(float);
  if ((rc = ensure(ctx, ctx->cl_mat, mat))) return rc;
  rc = wmd_pairwise_rmsd(ctx, coords, n_frames, n_atoms, stride, sel, n_sel, WMD_PAIR_RMS, mode,
                         static_cast<float*>(ctx->cl_mat.ptr), stream);
  if (rc) return rc;
  const size_t n = (size_t)n_frames;
  // device outputs: labels [n], sizes [n], centroids [n], cluster count, best sums [n]
  if ((rc = ensure(ctx, ctx->cl_scratch, wmd::dbscan_scratch_bytes(n_frames))) ||
      (rc = ensure(ctx, ctx->cl_out, n * (4 + 4 + 4 + 8) + 16)))
    return rc;
  char* o = static_cast<char*>(ctx->cl_out.ptr);
  int* dlabels = reinterpret_cast<int*>(o);
  unsigned* dsizes = reinterpret_cast<unsigned*>(o + n * 4);
  unsigned* dcent = reinterpret_cast<unsigned*>(o + n * 8);
  int* dcount = reinterpret_cast<int*>(o + n * 12);
  unsigned long long* dbest = reinterpret_cast<unsigned long long*>(o + ((n * 12 + 4 + 7) & ~size_t(7)));
  const float* D = static_cast<const float*>(ctx->cl_mat.ptr);
  CU(wmd::dbscan_run(D, n_frames, (double)eps, std::max<int64_t>(1, min_samples), ctx->cl_scratch.ptr, dlabels, dcount,
                     ctx->status_dev, ctx->sm_count, s),
     "dbscan");
  int count = 0;
  CU(cudaMemcpyAsync(&count, dcount, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
  CU(cudaStreamSynchronize(s), "synchronize");
  if ((rc = check_status(ctx))) return rc;
  CU(wmd::dbscan_summary(D, n_frames, dlabels, count, ctx->cl_scratch.ptr, dsizes, dcent, dbest, s), "dbscan summary");
  auto put = [&](void* dst, const void* src, size_t bytes) -> int {
    if (!bytes) return WMD_OK;
    CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s), "copy out");
    return WMD_OK;
  };
  if ((rc = put(labels, dlabels, n * 4)) || (rc = put(sizes, dsizes, (size_t)count * 4)) ||
      (rc = put(centroids, dcent, (size_t)count * 4)))
    return rc;
  CU(cudaStreamSynchronize(s), "synchronize");
  *n_clusters = count;
  return check_status(ctx);
}

static uint64_t km_xorshift64(uint64_t* state) {
  // xorshift64 as clustering.rs:536-547 writes it (zero state replaced)
  uint64_t x = *state;
  if (x == 0) x = 0x9E3779B97F4A7C15ull;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *state = x;
  return x;
}

WMD_EXPORT int wmd_cluster_kmeans(wmd_ctx* ctx, const float* coords, int64_t n_frames, int64_t n_atoms, int stride,
                                  const uint32_t* sel, int64_t n_sel, int64_t n_clusters, int64_t max_iter, float tol,
                                  uint64_t seed, int32_t* labels, uint32_t* centroids, uint32_t* sizes,
                                  int64_t* n_out, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!n_out) return set_err(ctx, WMD_ERR_INVALID_ARG, "n_out is null");
  *n_out = 0;
  if (n_sel == 0) return set_err(ctx, WMD_ERR_MISMATCH, "mismatch: trajectory_cluster requires a non-empty selection");
  if (stride != 3 && stride != 4) return set_err(ctx, WMD_ERR_INVALID_ARG, "stride must be 3 or 4 (got %d)", stride);
  if (n_frames < 0 || n_atoms < 0 || n_sel < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative size");
  if (n_frames > (int64_t)0x7fffffff) return set_err(ctx, WMD_ERR_UNSUPPORTED, "too many frames for clustering");
  if (!sel && n_sel > n_atoms)
    return set_err(ctx, WMD_ERR_MISMATCH, "selection of %lld atoms exceeds the frame's %lld atoms", (long long)n_sel,
                   (long long)n_atoms);
  if (n_frames > 0 && (!coords || !labels || !centroids || !sizes))
    return set_err(ctx, WMD_ERR_INVALID_ARG, "coords, labels, centroids and sizes are required");
  if (n_frames == 0) return WMD_OK;
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t N = n_frames, K = std::min<int64_t>(std::max<int64_t>(n_clusters, 1), N);
  const int64_t iters = std::max<int64_t>(max_iter, 1);
  const double tolerance = std::max(0.0, (double)tol);
  const int64_t nf = n_sel * 3;
  // frame 0's selected atoms are the reference (build_aligned_features,
  // clustering.rs:376-386)
  std::vector<float> f0((size_t)n_atoms * stride), ref((size_t)n_sel * 3);
  CU(cudaMemcpy(f0.data(), coords, f0.size() * sizeof(float), cudaMemcpyDefault), "read frame 0");
  std::vector<uint32_t> hsel;
  if (sel) {
    hsel.resize((size_t)n_sel);
    CU(cudaMemcpy(hsel.data(), sel, hsel.size() * 4, cudaMemcpyDefault), "read selection");
    for (uint32_t a : hsel)
      if ((int64_t)a >= n_atoms)
        return set_err(ctx, WMD_ERR_INVALID_ARG, "selection index %u out of range for %lld atoms", a, (long long)n_atoms);
  }
  for (int64_t a = 0; a < n_sel; ++a) {
    const int64_t atom = sel ? hsel[a] : a;
    for (int c = 0; c < 3; ++c) ref[a * 3 + c] = f0[atom * stride + c];
  }
  wmd_ref* r = nullptr;
  if ((rc = reference_upload(ctx, ref.data(), n_sel, 3, nullptr, &r))) return rc;
  struct RefFree {
    wmd_ctx* c;
    wmd_ref* r;
    ~RefFree() { wmd_reference_free(c, r); }
  } ref_guard{ctx, r};
  const uint32_t* dsel = nullptr;
  if ((rc = resolve_sel(ctx, sel, n_sel, n_atoms, &dsel, s))) return rc;
  const size_t feat_bytes = (size_t)N * nf * sizeof(double);
  if ((rc = ensure(ctx, ctx->km_feat, feat_bytes)) ||
      (rc = ensure(ctx, ctx->km_xf, (size_t)N * wmd::kStatDoubles * sizeof(double))))
    return rc;
  double* feat = static_cast<double*>(ctx->km_feat.ptr);
  double* xf_all = static_cast<double*>(ctx->km_xf.ptr);
  rc = for_each_chunk(ctx, coords, n_frames, n_atoms, stride, s, [&](const float* dc, int64_t fb, int64_t nfr) -> int {
    int r2 = superpose_device(ctx, dc, nfr, n_atoms, stride, dsel, r, 0, nullptr, nullptr, s, nullptr,
                              xf_all + fb * wmd::kStatDoubles);
    if (r2) return r2;
    CU(wmd::kmeans_features(dc, nfr, n_atoms, stride, dsel, n_sel, xf_all + fb * wmd::kStatDoubles,
                            feat + (size_t)fb * nf, ctx->sm_count, s),
       "kmeans features");
    return WMD_OK;
  });
  if (rc) return rc;
  // work: centers x2, sums [K][nf]; labels [N]; counts [K]; reseed [K]; shift [K];
  // dist [N]; best [K]; sizes, centroids [K]
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t cbytes = al((size_t)K * nf * 8);
  const size_t total = 3 * cbytes + al(N * 4) + al(K * 4) + al(K * 8) + al(K * 8) + al(N * 8) + al(K * 8) +
                       2 * al(K * 4);
  if ((rc = ensure(ctx, ctx->km_work, total))) return rc;
  char* w = static_cast<char*>(ctx->km_work.ptr);
  double* cen_a = reinterpret_cast<double*>(w);
  double* cen_b = reinterpret_cast<double*>(w + cbytes);
  double* sums = reinterpret_cast<double*>(w + 2 * cbytes);
  size_t off = 3 * cbytes;
  auto take = [&](size_t b) { char* p = w + off; off += al(b); return p; };
  int* dlabels = reinterpret_cast<int*>(take(N * 4));
  int* dcounts = reinterpret_cast<int*>(take(K * 4));
  int64_t* dreseed = reinterpret_cast<int64_t*>(take(K * 8));
  double* dshift = reinterpret_cast<double*>(take(K * 8));
  double* ddist = reinterpret_cast<double*>(take(N * 8));
  unsigned long long* dbest = reinterpret_cast<unsigned long long*>(take(K * 8));
  unsigned* dsizes = reinterpret_cast<unsigned*>(take(K * 4));
  unsigned* dcent = reinterpret_cast<unsigned*>(take(K * 4));
  // initial centers: the first K of a Fisher-Yates shuffle (clustering.rs:433-445, 527-534)
  uint64_t state = seed == 0 ? 0x9E3779B97F4A7C15ull : seed;
  std::vector<int64_t> order((size_t)N);
  for (int64_t i = 0; i < N; ++i) order[i] = i;
  for (int64_t i = N - 1; i >= 1; --i) {
    const int64_t j = (int64_t)(km_xorshift64(&state) % (uint64_t)(i + 1));
    std::swap(order[i], order[j]);
  }
  std::vector<int64_t> idx(order.begin(), order.begin() + K);
  CU(cudaMemcpyAsync(dreseed, idx.data(), (size_t)K * 8, cudaMemcpyHostToDevice, s), "upload");
  CU(wmd::kmeans_gather(feat, nf, dreseed, (int)K, cen_a, s), "kmeans init");
  std::vector<int> counts((size_t)K);
  std::vector<int64_t> reseed((size_t)K);
  std::vector<double> shift((size_t)K);
  for (int64_t it = 0; it < iters; ++it) {
    CU(wmd::kmeans_assign(feat, N, nf, cen_a, (int)K, dlabels, nullptr, s), "kmeans assign");
    CU(wmd::kmeans_sums(feat, N, nf, dlabels, (int)K, sums, dcounts, s), "kmeans sums");
    CU(cudaMemcpyAsync(counts.data(), dcounts, (size_t)K * 4, cudaMemcpyDeviceToHost, s), "D2H");
    CU(cudaStreamSynchronize(s), "synchronize");
    for (int64_t c = 0; c < K; ++c)
      reseed[c] = counts[c] == 0 ? (int64_t)(km_xorshift64(&state) % (uint64_t)N) : -1;
    CU(cudaMemcpyAsync(dreseed, reseed.data(), (size_t)K * 8, cudaMemcpyHostToDevice, s), "upload");
    CU(wmd::kmeans_centers(feat, nf, sums, dcounts, dreseed, (int)K, cen_a, cen_b, dshift, s), "kmeans centers");
    CU(cudaMemcpyAsync(shift.data(), dshift, (size_t)K * 8, cudaMemcpyDeviceToHost, s), "D2H");
    CU(cudaStreamSynchronize(s), "synchronize");
    std::swap(cen_a, cen_b);
    double max_shift = 0.0;
    for (double v : shift) max_shift = std::max(max_shift, v);
    if (max_shift <= tolerance) break;
  }
  CU(wmd::kmeans_finish(feat, N, nf, cen_a, dlabels, (int)K, ddist, dbest, dsizes, dcent, s), "kmeans finish");
  std::vector<unsigned> hs((size_t)K), hc((size_t)K);
  CU(cudaMemcpyAsync(hs.data(), dsizes, (size_t)K * 4, cudaMemcpyDeviceToHost, s), "D2H");
  CU(cudaMemcpyAsync(hc.data(), dcent, (size_t)K * 4, cudaMemcpyDeviceToHost, s), "D2H");
  CU(cudaMemcpyAsync(labels, dlabels, (size_t)N * 4, cudaMemcpyDefault, s), "copy out");
  CU(cudaStreamSynchronize(s), "synchronize");
  for (int64_t c = 0; c < K; ++c)
    if (hs[c] == 0) hc[c] = 0;  // the reference's best_idx default
  CU(cudaMemcpy(sizes, hs.data(), (size_t)K * 4, cudaMemcpyDefault), "copy out");
  CU(cudaMemcpy(centroids, hc.data(), (size_t)K * 4, cudaMemcpyDefault), "copy out");
  *n_out = K;
  return check_status(ctx);
}

// Builds the device trajectory table for a tile shape; returns total items
// (tile-major layout) and fills the frame-group partition (frame-major).
// Each trajectory's centred reference is followed by 32 zero atoms (the lanes
// forward copies whole 32-atom blocks of it), every block 16-byte aligned.
static int64_t batch_yc_doubles(int64_t n_atoms) { return (n_atoms * 3 + 1) / 2 * 2 + 32 * 3; }

static int64_t build_segs(const std::vector<wmd_batch_desc>& d, int apt, double* yc_base, bool with_grad,
                          std::vector<wmd::BatchSeg>& segs, int64_t* total_frames, int64_t* total_groups,
                          int64_t* total_cost, int64_t* total_lane_cost) {
  const int tile = wmd::batched_tile_atoms(apt);
  segs.assign(d.size(), wmd::BatchSeg{});
  int64_t items = 0, frames = 0, yoff = 0, groups = 0, cost = 0, lane_cost = 0;
  for (size_t i = 0; i < d.size(); ++i) {
    wmd::BatchSeg& g = segs[i];
    g.coords = d[i].coords;
    g.ref = d[i].ref;
    g.rmsd = d[i].rmsd;
    g.grad = d[i].grad;
    g.n_atoms = d[i].n_atoms;
    g.n_frames = d[i].n_frames;
    g.n_tiles = (int)((d[i].n_atoms + tile - 1) / tile);
    g.yc = yc_base + yoff;
    yoff += batch_yc_doubles(d[i].n_atoms);
    // lanes layout: (tile, 32-frame group) units, tile-major; cost ~ the
    // tile's atom-frames plus a per-stage overhead of about 8 atoms' work and a
    // per-unit one of about a stage (the partial records); the last tile holds
    // the remainder of the atoms
    g.lane_cost0 = lane_cost;
    auto unit_cost = [](int64_t at) { return 32 * (at + 8 * ((at + 31) / 32) + 32); };
    if (g.n_atoms > 0 && g.n_frames > 0) {
      const int64_t groups_f = (g.n_frames + 31) / 32;
      g.lane_units = (int64_t)g.n_tiles * groups_f;
      g.lane_full_units = (int64_t)(g.n_tiles - 1) * groups_f;
      g.lane_unit_cost = unit_cost(tile);
      g.lane_last_cost = unit_cost(g.n_atoms - (int64_t)(g.n_tiles - 1) * tile);
    } else {
      g.lane_units = g.lane_full_units = 0;
      g.lane_unit_cost = g.lane_last_cost = 1;
    }
    lane_cost += g.lane_full_units * g.lane_unit_cost + (g.lane_units - g.lane_full_units) * g.lane_last_cost;
    g.item0 = items;
    g.frame0 = frames;
    items += (int64_t)g.n_tiles * g.n_frames;
    frames += g.n_frames;
    // frame groups
    g.group0 = groups;
    g.cost0 = cost;
    if (g.n_atoms > 0 && g.n_frames > 0) {
      const int64_t fb = g.n_atoms * 12;
      g.m_group = (int)std::max<int64_t>(1, std::min<int64_t>(wmd::kGroupFrames, wmd::kGroupBytes / fb));
      g.n_groups = (g.n_frames + g.m_group - 1) / g.m_group;
      const int64_t passes = (with_grad && g.grad) ? 2 : 1;
      const int64_t frame_cost = (int64_t)g.n_tiles * passes * wmd::kCostItem;
      g.group_cost = g.m_group * frame_cost + wmd::kCostFinish;
      const int64_t last = g.n_frames - (g.n_groups - 1) * g.m_group;
      groups += g.n_groups;
      cost += (g.n_groups - 1) * g.group_cost + last * frame_cost + wmd::kCostFinish;
    } else {
      g.m_group = 1;
      g.n_groups = 0;
      g.group_cost = 1;
    }
  }
  *total_frames = frames;
  *total_groups = groups;
  *total_cost = cost;
  *total_lane_cost = lane_cost;
  return items;
}

WMD_EXPORT int wmd_batched_prepare(wmd_ctx* ctx, const wmd_batch_desc* descs, int n_traj, int with_grad) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (n_traj < 0 || (n_traj > 0 && !descs)) return set_err(ctx, WMD_ERR_INVALID_ARG, "invalid batch");
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  ctx->b_ready = false;
  std::vector<wmd_batch_desc> d(descs, descs + n_traj);
  int64_t sum_atoms = 0;
  for (int i = 0; i < n_traj; ++i) {
    wmd_batch_desc& x = d[i];
    if (x.n_atoms < 0 || x.n_frames < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "trajectory %d: negative size", i);
    if (x.n_frames == 0) {
      x.n_atoms = 0;  // nothing to read or write
      continue;
    }
    if (!x.rmsd || classify(x.rmsd) != Mem::Device)
      return set_err(ctx, WMD_ERR_INVALID_ARG, "trajectory %d: rmsd must be device memory", i);
    if (x.n_atoms == 0) continue;  // RMSD 0 per frame, like an empty selection
    if (!x.coords || !x.ref) return set_err(ctx, WMD_ERR_INVALID_ARG, "trajectory %d: coords and ref are required", i);
    if (classify(x.coords) != Mem::Device || classify(x.ref) != Mem::Device ||
        (x.grad && classify(x.grad) != Mem::Device))
      return set_err(ctx, WMD_ERR_INVALID_ARG, "trajectory %d: batched buffers must be device memory", i);
    if (reinterpret_cast<uintptr_t>(x.coords) & 15u)
      return set_err(ctx, WMD_ERR_INVALID_ARG, "trajectory %d: coords must be 16-byte aligned", i);
    if (with_grad && (reinterpret_cast<uintptr_t>(x.grad) & 15u))
      return set_err(ctx, WMD_ERR_INVALID_ARG, "trajectory %d: grad must be 16-byte aligned", i);
    if (!with_grad) x.grad = nullptr;
  }
  for (int i = 0; i < n_traj; ++i) sum_atoms += batch_yc_doubles(d[i].n_atoms);
  int64_t frames4 = 0, frames8 = 0;
  std::vector<wmd::BatchSeg> s4, s8;
  if ((rc = ensure(ctx, ctx->b_yc, (size_t)std::max<int64_t>(sum_atoms, 2) * sizeof(double)))) return rc;
  double* yc = static_cast<double*>(ctx->b_yc.ptr);
  // the padding after every block must read as zeros
  CU(cudaMemset(yc, 0, (size_t)std::max<int64_t>(sum_atoms, 2) * sizeof(double)), "memset");
  int64_t groups4 = 0, groups8 = 0, cost4 = 0, cost8 = 0, lcost4 = 0, lcost8 = 0;
  const int64_t items4 = build_segs(d, 4, yc, with_grad != 0, s4, &frames4, &groups4, &cost4, &lcost4);
  const int64_t items8 = build_segs(d, 8, yc, with_grad != 0, s8, &frames8, &groups8, &cost8, &lcost8);
  const int64_t frames = frames4;
  const size_t rec = wmd::kStatDoubles * sizeof(double);
  // the lanes layout's tensor maps (one per trajectory; the same for both tile shapes)
  {
    std::vector<CUtensorMap> maps((size_t)std::max(n_traj, 1));
    std::string msg;
    if (!wmd::batched_encode_maps(s8, maps.data(), &msg)) return set_err(ctx, WMD_ERR_CUDA, "%s", msg.c_str());
    for (size_t i = 0; i < s4.size(); ++i) s4[i].tma = s8[i].tma;
    if ((rc = ensure(ctx, ctx->b_maps, maps.size() * sizeof(CUtensorMap)))) return rc;
    CU(cudaMemcpy(ctx->b_maps.ptr, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice),
       "upload tensor maps");
  }
  if ((rc = ensure(ctx, ctx->b_segs, std::max<size_t>(1, (size_t)n_traj) * sizeof(wmd::BatchSeg))) ||
      (rc = ensure(ctx, ctx->b_partial, (size_t)std::max<int64_t>(1, std::max(items4, items8)) * rec)) ||
      (rc = ensure(ctx, ctx->b_refine, (size_t)std::max<int64_t>(1, frames) * rec)) ||
      (rc = ensure(ctx, ctx->b_count, sizeof(unsigned), true)))
    return rc;
  if (with_grad && (rc = ensure(ctx, ctx->b_rot, (size_t)std::max<int64_t>(1, frames) * rec))) return rc;
  wmd::BatchPlan P;
  P.n_segs = n_traj;
  P.segs_dev = static_cast<wmd::BatchSeg*>(ctx->b_segs.ptr);
  P.launch.segs = P.segs_dev;
  P.launch.maps = static_cast<const CUtensorMap*>(ctx->b_maps.ptr);
  P.launch.n_segs = n_traj;
  P.launch.total_frames = frames;
  P.launch.partial = static_cast<double*>(ctx->b_partial.ptr);
  P.launch.rot = with_grad ? static_cast<double*>(ctx->b_rot.ptr) : nullptr;
  P.launch.refine = static_cast<double*>(ctx->b_refine.ptr);
  P.launch.refine_count = static_cast<unsigned*>(ctx->b_count.ptr);
  P.launch.status = ctx->status_dev;
  // Autotuner: time the whole pipeline once per candidate layout (tile-major
  // or frame-major) and tile shape (512 or 1024 atoms) on this batch.
  // WARPMD_BATCHED_LAYOUT=tiles|frames and WARPMD_BATCHED_TILE_ATOMS=512|1024
  // pin either choice.
  auto configure = [&](int variant, int apt) -> int {
    std::vector<wmd::BatchSeg>& sv = apt == 4 ? s4 : s8;
    if (n_traj > 0)
      CU(cudaMemcpy(P.segs_dev, sv.data(), sv.size() * sizeof(wmd::BatchSeg), cudaMemcpyHostToDevice), "upload");
    P.variant = variant;
    P.apt = apt;
    P.launch.total_items = apt == 4 ? items4 : items8;
    P.launch.total_groups = apt == 4 ? groups4 : groups8;
    P.launch.total_cost = apt == 4 ? cost4 : cost8;
    P.launch.total_lane_cost = apt == 4 ? lcost4 : lcost8;
    if (variant == wmd::kBatchLanes) {
      int64_t units = 0;
      for (const wmd::BatchSeg& g : sv) units += g.lane_units;
      P.grid_fwd = wmd::batched_lanes_grid(ctx->sm_count, units);
      P.grid_bwd = wmd::batched_grid(apt, true, ctx->sm_count, P.launch.total_items);
    } else if (variant == wmd::kBatchFrames) {
      P.grid_fwd = wmd::batched_frame_grid(apt, with_grad != 0, ctx->sm_count, P.launch.total_groups);
      P.grid_bwd = P.grid_fwd;
    } else {
      P.grid_fwd = wmd::batched_grid(apt, false, ctx->sm_count, P.launch.total_items);
      P.grid_bwd = wmd::batched_grid(apt, true, ctx->sm_count, P.launch.total_items);
    }
    return WMD_OK;
  };
  std::vector<int> apts = {8, 4}, layouts = {wmd::kBatchFrames, wmd::kBatchTiles, wmd::kBatchLanes};
  if (const char* env = std::getenv("WARPMD_BATCHED_TILE_ATOMS")) {
    if (std::strcmp(env, "512") == 0) apts = {4};
    else if (std::strcmp(env, "1024") == 0) apts = {8};
  }
  if (const char* env = std::getenv("WARPMD_BATCHED_LAYOUT")) {
    if (std::strcmp(env, "tiles") == 0) layouts = {wmd::kBatchTiles};
    else if (std::strcmp(env, "frames") == 0) layouts = {wmd::kBatchFrames};
    else if (std::strcmp(env, "lanes") == 0) layouts = {wmd::kBatchLanes};
  }
  float best_ms = -1.f;
  int best_apt = apts[0], best_layout = layouts[0];
  if (n_traj > 0 && apts.size() * layouts.size() > 1) {
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0), "event");
    CU(cudaEventCreate(&e1), "event");
    for (int layout : layouts)
      for (int apt : apts) {
        if ((rc = configure(layout, apt))) return rc;
        CU(wmd::batched_enqueue(P, with_grad != 0, 0), "batched warm-up");
        CU(cudaEventRecord(e0, 0), "event");
        CU(wmd::batched_enqueue(P, with_grad != 0, 0), "batched tuning run");
        CU(cudaEventRecord(e1, 0), "event");
        CU(cudaEventSynchronize(e1), "synchronize");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best_ms < 0.f || ms < best_ms) {
          best_ms = ms;
          best_apt = apt;
          best_layout = layout;
        }
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if ((rc = configure(best_layout, best_apt))) return rc;
  if ((rc = check_status(ctx))) return rc;
  ctx->b_plan = P;
  ctx->b_descs.assign(descs, descs + n_traj);
  ctx->b_grad = with_grad != 0;
  ctx->b_ready = true;
  return WMD_OK;
}

WMD_EXPORT int wmd_batched_rmsd(wmd_ctx* ctx, const wmd_batch_desc* descs, int n_traj, int with_grad, void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if (!ctx->b_ready || n_traj != (int)ctx->b_descs.size() || (with_grad && !ctx->b_grad) ||
      (n_traj > 0 && std::memcmp(descs, ctx->b_descs.data(), sizeof(wmd_batch_desc) * (size_t)n_traj) != 0))
    return set_err(ctx, WMD_ERR_INVALID_ARG,
                   "wmd_batched_rmsd needs the same descriptors wmd_batched_prepare was called with");
  if (n_traj == 0) return WMD_OK;
  CU(wmd::batched_enqueue(ctx->b_plan, with_grad != 0, static_cast<cudaStream_t>(stream)), "batched launch");
  return WMD_OK;
}

WMD_EXPORT int wmd_batched_layout(const wmd_ctx* ctx, int* tile_atoms, int* frame_major) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!ctx->b_ready) return set_err(const_cast<wmd_ctx*>(ctx), WMD_ERR_INVALID_ARG, "no batch is prepared");
  if (tile_atoms) *tile_atoms = wmd::batched_tile_atoms(ctx->b_plan.apt);
  if (frame_major) *frame_major = ctx->b_plan.variant;
  return WMD_OK;
}

// ---------------------------------------------------------------------------
// DCD trajectories (DcdReader, crates/traj-io/src/dcd.rs; PyTrajectory
// open_dcd / read_chunk, crates/traj-py/src/io.rs:687-708, 1335-1560)
// ---------------------------------------------------------------------------

struct wmd_dcd {
  wmd::DcdFile f;
  int device = 0;
  std::unique_ptr<wmd::ReadPool> pool;  // parallel preads per batch
  HostBuf pin[2];   // raw file bytes of a batch (+ the X-offset table of an indexed file)
  DevBuf raw[2], coords;
  cudaEvent_t h2d_done[2] = {nullptr, nullptr};
  cudaEvent_t consumed[2] = {nullptr, nullptr};
};

namespace {

// Raw bytes per batch: large enough to keep the copy engine and the pread
// threads streaming, small enough that two pinned slots stay cheap.
constexpr int64_t kDcdBatchBytes = int64_t(64) << 20;

int dcd_err(wmd_ctx* ctx, const wmd::DcdError& e) {
  const int code = e.kind == wmd::kDcdIo ? WMD_ERR_IO : e.kind == wmd::kDcdParse ? WMD_ERR_PARSE : WMD_ERR_UNSUPPORTED;
  const char* cls = e.kind == wmd::kDcdIo ? "io error" : e.kind == wmd::kDcdParse ? "parse error" : "unsupported";
  return set_err(ctx, code, "%s: %s", cls, e.msg.c_str());
}

// Status of the decode launches: a record marker that broke the layout
// assumed for the file is returned in *bad_record, anything else as an error.
int dcd_status(wmd_ctx* ctx, bool* bad_record) {
  const int st = __atomic_exchange_n(ctx->status_host, 0, __ATOMIC_ACQ_REL);
  *bad_record = (st & wmd::kStatusBadRecord) != 0;
  const int rest = st & ~wmd::kStatusBadRecord;
  if (!rest) return WMD_OK;
  if (rest & wmd::kStatusBadIndex)
    return set_err(ctx, WMD_ERR_MISMATCH, "mismatch: selection index out of bounds (device selection)");
  return set_err(ctx, WMD_ERR_TIMEOUT, "a device-side wait exceeded its limit (status 0x%x)", rest);
}

// Host selection indices checked as validate_selection does
// (crates/traj-io/src/selection_support.rs:3-13).
int dcd_check_sel(wmd_ctx* ctx, const wmd::DcdFile& F, const uint32_t* sel, int64_t n_sel) {
  if (!sel || classify(sel) == Mem::Device) return WMD_OK;
  for (int64_t i = 0; i < n_sel; ++i)
    if ((int64_t)sel[i] >= F.n_atoms)
      return set_err(ctx, WMD_ERR_MISMATCH, "mismatch: selection index %u out of bounds for trajectory with %lld atoms",
                     sel[i], (long long)F.n_atoms);
  return WMD_OK;
}

// Streams frames [first, first + n) through the two pinned and device slots.
// Per batch: pread (host threads) -> on_host(pinned bytes, their file offset,
// frames [fa, fb)) -> host->device copy (copy stream) -> decode (stream s)
// into dout at the batch's frames, or into scratch when dout is null ->
// on_dev(decoded frames, fa - first, fb - fa).  The pread of batch k + 1 runs
// while batch k is copied and decoded.
template <class HostFn, class DevFn>
int dcd_stream(wmd_ctx* ctx, wmd_dcd* d, int64_t first, int64_t n, const uint32_t* dsel, int64_t n_out, float* dout,
               cudaStream_t s, HostFn on_host, DevFn on_dev) {
  const wmd::DcdFile& F = d->f;
  if (n == 0) return WMD_OK;
  std::vector<int64_t> cuts{first};
  size_t max_bytes = 0;
  int64_t max_frames = 0;
  for (int64_t a = first; a < first + n;) {
    int64_t b;
    if (!F.indexed) {
      b = std::min(first + n, a + std::max<int64_t>(1, kDcdBatchBytes / F.stride));
    } else {
      b = a + 1;
      while (b < first + n && F.frame_begin(b + 1) - F.frame_begin(a) <= kDcdBatchBytes) ++b;
    }
    const int64_t base = F.frame_begin(a) & ~int64_t(15);
    const size_t padded = ((size_t)(F.frame_begin(b) - base) + 15) & ~size_t(15);
    max_bytes = std::max(max_bytes, padded + (F.indexed ? (size_t)(b - a) * 8 : 0));
    max_frames = std::max(max_frames, b - a);
    cuts.push_back(b);
    a = b;
  }
  int rc;
  for (int k = 0; k < 2; ++k) {
    if ((rc = ensure_host(ctx, d->pin[k], max_bytes))) return rc;
    if ((rc = ensure(ctx, d->raw[k], max_bytes))) return rc;
  }
  float* scratch = nullptr;
  if (!dout) {
    if ((rc = ensure(ctx, d->coords, (size_t)max_frames * (size_t)n_out * 3 * sizeof(float)))) return rc;
    scratch = static_cast<float*>(d->coords.ptr);
  }
  for (int k = 0; k < 2; ++k) {
    CU(cudaEventRecord(d->consumed[k], s), "event");
    CU(cudaEventRecord(d->h2d_done[k], ctx->copy_stream), "event");
  }
  for (size_t k = 0; k + 1 < cuts.size(); ++k) {
    const int b = (int)(k & 1);
    const int64_t fa = cuts[k], fb = cuts[k + 1], nf = fb - fa;
    const int64_t base = F.frame_begin(fa) & ~int64_t(15);
    const int64_t bytes = F.frame_begin(fb) - base;
    const size_t padded = ((size_t)bytes + 15) & ~size_t(15);
    CU(cudaEventSynchronize(d->h2d_done[b]), "pinned slot wait");
    uint8_t* hp = static_cast<uint8_t*>(d->pin[b].ptr);
    if (wmd::DcdError e = wmd::dcd_pread(F, *d->pool, hp, base, bytes)) return dcd_err(ctx, e);
    size_t copy = padded;
    if (F.indexed) {
      int64_t* tab = reinterpret_cast<int64_t*>(hp + padded);
      for (int64_t f = 0; f < nf; ++f) tab[f] = F.frame_x(fa + f);
      copy += (size_t)nf * 8;
    }
    on_host(static_cast<const uint8_t*>(hp), base, fa, fb);
    CU(cudaStreamWaitEvent(ctx->copy_stream, d->consumed[b], 0), "stream wait");
    CU(cudaMemcpyAsync(d->raw[b].ptr, hp, copy, cudaMemcpyHostToDevice, ctx->copy_stream), "H2D");
    CU(cudaEventRecord(d->h2d_done[b], ctx->copy_stream), "event");
    CU(cudaStreamWaitEvent(s, d->h2d_done[b], 0), "stream wait");
    wmd::DcdDecode D;
    D.raw = static_cast<const uint8_t*>(d->raw[b].ptr);
    D.raw_off = base;
    D.first = fa;
    D.n_frames = nf;
    D.xoff = F.indexed ? reinterpret_cast<const int64_t*>(static_cast<const uint8_t*>(d->raw[b].ptr) + padded) : nullptr;
    D.data_start = F.data_start;
    D.stride = F.stride;
    D.cell = F.cell;
    D.n_atoms = F.n_atoms;
    D.marker = F.marker;
    D.big = F.big;
    D.aligned = (F.data_start & 3) == 0;
    D.scale = F.length_scale;
    D.sel = dsel;
    D.n_out = n_out;
    D.out = dout ? dout + (size_t)(fa - first) * (size_t)n_out * 3 : scratch;
    D.status = ctx->status_dev;
    CU(wmd::launch_dcd_decode(D, ctx->sm_count, s), "dcd decode launch");
    if ((rc = on_dev(D.out, fa - first, nf))) return rc;
    CU(cudaEventRecord(d->consumed[b], s), "event");
  }
  return WMD_OK;
}

// Frames a read from `first` of up to max_frames returns, or the error of a
// damaged end of file that the read would reach.
int dcd_span(wmd_ctx* ctx, const wmd::DcdFile& F, int64_t first, int64_t max_frames, int64_t* n) {
  const int64_t avail = std::max<int64_t>(0, F.n_frames - first);
  *n = std::min(max_frames, avail);
  if (max_frames > avail && F.end) return dcd_err(ctx, F.end);
  return WMD_OK;
}

}  // namespace

WMD_EXPORT int wmd_dcd_open(wmd_ctx* ctx, const char* path, float length_scale, wmd_dcd** out) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (!out || !path) return set_err(ctx, WMD_ERR_INVALID_ARG, "path or out is null");
  *out = nullptr;
  DeviceGuard g(ctx->device);
  wmd_dcd* d = new wmd_dcd();
  d->device = ctx->device;
  if (wmd::DcdError e = wmd::dcd_open(path, length_scale, &d->f)) {
    wmd::dcd_close(&d->f);
    delete d;
    return dcd_err(ctx, e);
  }
  const unsigned hw = std::thread::hardware_concurrency();
  int threads = (int)std::max(1u, std::min(16u, hw ? hw : 1u));
  if (const char* v = std::getenv("WMD_DCD_THREADS")) {  // pread threads per batch
    const int t = std::atoi(v);
    if (t > 0 && t <= 64) threads = t;
  }
  try {  // nothing may throw across the C ABI
    d->pool.reset(new wmd::ReadPool(threads));
  } catch (...) {
    wmd::dcd_close(&d->f);
    delete d;
    return set_err(ctx, WMD_ERR_OOM, "could not allocate the file reader");
  }
  for (int k = 0; k < 2; ++k) {
    cudaError_t e = cudaEventCreateWithFlags(&d->h2d_done[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d->consumed[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
      wmd_dcd_close(ctx, d);
      return cuda_err(ctx, e, "event");
    }
  }
  *out = d;
  return WMD_OK;
}

WMD_EXPORT int wmd_dcd_close(wmd_ctx* ctx, wmd_dcd* d) {
  if (!d) return WMD_OK;
  DeviceGuard g(d->device);
  for (int k = 0; k < 2; ++k) {
    if (d->h2d_done[k]) {
      cudaEventSynchronize(d->h2d_done[k]);
      cudaEventDestroy(d->h2d_done[k]);
    }
    if (d->consumed[k]) {
      cudaEventSynchronize(d->consumed[k]);
      cudaEventDestroy(d->consumed[k]);
    }
  }
  for (DevBuf* b : {&d->raw[0], &d->raw[1], &d->coords})
    if (b->ptr) cudaFree(b->ptr);
  for (HostBuf* b : {&d->pin[0], &d->pin[1]})
    if (b->ptr) cudaFreeHost(b->ptr);
  wmd::dcd_close(&d->f);
  delete d;
  (void)ctx;
  return WMD_OK;
}

WMD_EXPORT int wmd_dcd_info(const wmd_dcd* d, int64_t* n_atoms, int64_t* n_frames, int64_t* header_frames) {
  if (!d) return WMD_ERR_INVALID_ARG;
  if (n_atoms) *n_atoms = d->f.n_atoms;
  if (n_frames) *n_frames = d->f.n_frames;
  if (header_frames) *header_frames = d->f.header_frames;
  return WMD_OK;
}

WMD_EXPORT int wmd_dcd_read(wmd_ctx* ctx, wmd_dcd* d, int64_t first, int64_t max_frames, const uint32_t* sel,
                            int64_t n_sel, float* coords, int32_t* box_kind, float* box, int64_t* n_read,
                            void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (n_read) *n_read = 0;
  if (!d) return set_err(ctx, WMD_ERR_INVALID_ARG, "dcd is null");
  if (first < 0 || max_frames < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative frame range");
  if (sel && n_sel <= 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "atom_indices must not be empty");
  if ((box_kind && classify(box_kind) == Mem::Device) || (box && classify(box) == Mem::Device))
    return set_err(ctx, WMD_ERR_INVALID_ARG, "box outputs must be host memory");
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if ((rc = dcd_check_sel(ctx, d->f, sel, n_sel))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const wmd::DcdFile& F = d->f;
  const int64_t n_out = sel ? n_sel : F.n_atoms;
  const Mem cm = classify(coords);
  float* dout = cm == Mem::Device ? coords : nullptr;
  int64_t n_cap = max_frames;  // a retry never writes more frames than the first attempt sized
  for (int attempt = 0; attempt < 2; ++attempt) {
    int64_t n = 0;
    if ((rc = dcd_span(ctx, F, first, max_frames, &n))) return rc;
    n = std::min(n, n_cap);
    n_cap = n;
    if (n == 0) return WMD_OK;
    if (!coords) return set_err(ctx, WMD_ERR_INVALID_ARG, "coords is null");
    const uint32_t* dsel = nullptr;
    if ((rc = resolve_sel(ctx, sel, n_sel, F.n_atoms, &dsel, s))) return rc;
    auto on_host = [&](const uint8_t* hp, int64_t base, int64_t fa, int64_t fb) {
      if (!box_kind && !box) return;
      for (int64_t f = fa; f < fb; ++f) {
        float m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        int kind = 0;
        const int64_t c = F.frame_cell(f);
        if (c) kind = wmd::dcd_box(F, hp + (F.frame_begin(f) + F.marker - base), c, m);
        if (box_kind) box_kind[f - first] = kind;
        if (box) std::memcpy(box + (f - first) * 9, m, sizeof(m));
      }
    };
    auto on_dev = [&](const float* dc, int64_t f0, int64_t nf) -> int {
      if (dout) return WMD_OK;
      CU(cudaMemcpyAsync(coords + (size_t)f0 * (size_t)n_out * 3, dc, (size_t)nf * (size_t)n_out * 3 * sizeof(float),
                         cudaMemcpyDeviceToHost, s),
         "D2H");
      return WMD_OK;
    };
    if ((rc = dcd_stream(ctx, d, first, n, dsel, n_out, dout, s, on_host, on_dev))) return rc;
    CU(cudaStreamSynchronize(s), "synchronize");
    bool bad = false;
    if ((rc = dcd_status(ctx, &bad))) return rc;
    if (!bad) {
      if (n_read) *n_read = n;
      return WMD_OK;
    }
    if (F.indexed) break;
    wmd::dcd_index(&d->f);  // frames differ from the first one: read them by their own layout
  }
  return set_err(ctx, WMD_ERR_PARSE, "parse error: record markers disagree with the frame index");
}

WMD_EXPORT int wmd_dcd_rmsd(wmd_ctx* ctx, wmd_dcd* d, int64_t first, int64_t max_frames, const uint32_t* sel,
                            int64_t n_sel, const wmd_ref* ref, int align, double* out, int64_t* n_read,
                            void* stream) {
  if (!ctx) return WMD_ERR_INVALID_ARG;
  if (n_read) *n_read = 0;
  if (!d) return set_err(ctx, WMD_ERR_INVALID_ARG, "dcd is null");
  if (!ref) return set_err(ctx, WMD_ERR_INVALID_ARG, "reference is null");
  if (ref->info.w)
    return set_err(ctx, WMD_ERR_INVALID_ARG, "a weighted reference serves the superposition entry points only");
  if (first < 0 || max_frames < 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "negative frame range");
  if (sel && n_sel <= 0) return set_err(ctx, WMD_ERR_INVALID_ARG, "atom_indices must not be empty");
  const wmd::DcdFile& F = d->f;
  const int64_t n_out = sel ? n_sel : F.n_atoms;
  if (n_out != ref->info.n_sel)
    return set_err(ctx, WMD_ERR_MISMATCH, "reference has %lld atoms but the selection has %lld",
                   (long long)ref->info.n_sel, (long long)n_out);
  DeviceGuard g(ctx->device);
  int rc = check_status(ctx);
  if (rc) return rc;
  if ((rc = dcd_check_sel(ctx, F, sel, n_sel))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool oh = is_host(classify(out));
  int64_t n_cap = max_frames;
  for (int attempt = 0; attempt < 2; ++attempt) {
    int64_t n = 0;
    if ((rc = dcd_span(ctx, F, first, max_frames, &n))) return rc;
    n = std::min(n, n_cap);
    n_cap = n;
    if (n == 0) return WMD_OK;
    if (!out) return set_err(ctx, WMD_ERR_INVALID_ARG, "out is null");
    const uint32_t* dsel = nullptr;
    if ((rc = resolve_sel(ctx, sel, n_sel, F.n_atoms, &dsel, s))) return rc;
    double* o = out;
    if (oh) {
      if ((rc = ensure(ctx, ctx->out_tmp, (size_t)n * sizeof(double)))) return rc;
      o = static_cast<double*>(ctx->out_tmp.ptr);
    }
    auto on_host = [](const uint8_t*, int64_t, int64_t, int64_t) {};
    auto on_dev = [&](const float* dc, int64_t f0, int64_t nf) -> int {
      wmd::FrameOutputs fo;
      fo.rmsd = o + f0;
      return forward_device(ctx, dc, nf, n_out, 3, nullptr, ref, align, fo, s);
    };
    if ((rc = dcd_stream(ctx, d, first, n, dsel, n_out, nullptr, s, on_host, on_dev))) return rc;
    if (oh) CU(cudaMemcpyAsync(out, o, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H");
    CU(cudaStreamSynchronize(s), "synchronize");
    bool bad = false;
    if ((rc = dcd_status(ctx, &bad))) return rc;
    if (!bad) {
      if (n_read) *n_read = n;
      return WMD_OK;
    }
    if (F.indexed) break;
    wmd::dcd_index(&d->f);
  }
  return set_err(ctx, WMD_ERR_PARSE, "parse error: record markers disagree with the frame index");
}

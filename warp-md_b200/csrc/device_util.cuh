// device_util.cuh -- sm_100a primitives used by the RMSD kernels: mbarrier
// pipelines fed by 1-D bulk async copies (cp.async.bulk, the untiled TMA form,
// no multicast), bounded waits, and warp/CTA reductions of FP64 vectors.
#pragma once

#include <cstdint>

namespace wmd {

// A device-side wait gives up after this long and reports WMD_ERR_TIMEOUT
// through the context's status word instead of spinning forever.
constexpr uint64_t kWaitLimitNs = 4000000000ull;

// Limits of a launch's bounded device waits.  limit_ns replaces the default
// for the waits of a pipeline's consumers (exit-time drains of copies in
// flight keep kWaitLimitNs).  withhold != 0 is the error path's test: the
// producer serving the first consumer of CTA 0 arms nothing and copies
// nothing for its first stage, so that wait can only run out.  The kernels
// that honour it are the per-frame streaming forward kernels and the
// tensor-core pairwise kernel.
struct WaitCfg {
  uint64_t limit_ns = kWaitLimitNs;
  int withhold = 0;
};

enum DeviceStatus : int {
  kStatusOk = 0,
  kStatusTimeoutFull = 1,   // consumer waited too long for a copy to land
  kStatusTimeoutEmpty = 2,  // producer waited too long for a stage to drain
  kStatusTimeoutDrain = 4,  // exit-time wait for copies in flight ran out
  kStatusTimeoutPeer = 8,   // wait on another CTA's flag ran out
  kStatusBadIndex = 16,     // a selection index was >= n_atoms
  kStatusBadRecord = 64,    // a DCD record marker differs from the layout assumed for the file
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  // make the initialised barriers visible to the async (bulk-copy) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t tx_bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(tx_bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete.  Returns false (and
// records `code` in *status) when limit_ns passes first, or when *abort (a
// CTA-shared flag) is raised by another thread of the block.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status, int code,
                                          volatile int* abort, uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 0) {
      if (*abort) return false;
      if (global_timer_ns() - t0 > limit_ns) {
        if (status) atomicOr(status, code);
        *abort = 1;
        return false;
      }
    }
  }
}

// Exit-time wait for a stage's copies to land (phase `parity` of `bar`):
// a CTA must not exit while copies into its shared memory are in flight.
// Gives up after kWaitLimitNs, recording kStatusTimeoutDrain.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity, int* status) {
  const uint64_t t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_timer_ns() - t0 > kWaitLimitNs) {
      if (status) atomicOr(status, kStatusTimeoutDrain);
      return;
    }
  }
}

// 1-D bulk async copy global -> shared (TMA, untiled), completion signalled on
// `bar` as transaction bytes.  dst and src 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// 1-D bulk async copy shared -> global (TMA, untiled), tracked by bulk groups.
// dst and src 16-byte aligned, bytes % 16 == 0.  The writing threads must
// execute fence.proxy.async.shared::cta before the issuing thread reads the
// shared data through the async proxy.
__device__ __forceinline__ void bulk_copy_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until at most N committed bulk groups still read their shared source.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// Waits until at most N committed bulk groups are incomplete (writes done).
template <int N>
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void named_barrier_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Reduce-scatter of 16 doubles across a warp (butterfly): afterwards lane L holds
// the warp-wide sum of element (L >> 1) & 15 (lanes 2e and 2e+1 both hold e).
// 16 shuffles of doubles instead of 16 x 5 for a plain all-reduce.
__device__ __forceinline__ double warp_reduce_scatter16(double (&v)[16]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  {
    const bool hi = (lane >> 4) & 1;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double send = hi ? v[i] : v[i + 8];
      const double keep = hi ? v[i + 8] : v[i];
      v[i] = keep + __shfl_xor_sync(full, send, 16);
    }
  }
  {
    const bool hi = (lane >> 3) & 1;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double send = hi ? v[i] : v[i + 4];
      const double keep = hi ? v[i + 4] : v[i];
      v[i] = keep + __shfl_xor_sync(full, send, 8);
    }
  }
  {
    const bool hi = (lane >> 2) & 1;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double send = hi ? v[i] : v[i + 2];
      const double keep = hi ? v[i + 2] : v[i];
      v[i] = keep + __shfl_xor_sync(full, send, 4);
    }
  }
  {
    const bool hi = (lane >> 1) & 1;
    const double send = hi ? v[0] : v[1];
    const double keep = hi ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(full, send, 2);
  }
  return v[0] + __shfl_xor_sync(full, v[0], 1);
}

}  // namespace wmd

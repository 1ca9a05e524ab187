// Bulk asynchronous copies into shared memory with mbarrier completion
// (cp.async.bulk, single-CTA copies: a block copies only from this GPU's
// global memory into its own shared memory), and the fused PBiCGStab prologue
// shared by the streamed ILU substitution kernels.
#pragma once

#include <cstdint>

#include "devmath.cuh"
#include "krylov.hpp"

namespace gr {
namespace dev {

// Polls of an mbarrier before a wait gives up and reports GR_ETIMEOUT.
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fenceBarrierInit() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbarExpectTx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulkLoad(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait that lets the thread sleep until the phase completes or about
// `hintNs` nanoseconds pass, instead of returning at once: a waiting warp
// then takes no issue slots from the warps that do work.
__device__ __forceinline__ bool mbarTryWaitSleep(uint32_t bar, uint32_t parity, uint32_t hintNs) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(hintNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globalTimerNs() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Longest wait for one mbarrier phase before a kernel reports GR_ETIMEOUT.
constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s
// Bounded sleeping wait for the phase of `bar` with the given parity: true
// once it has completed; false after kWaitNs, after kWaitLimit sleeps, or
// (when `abort` is given) once *abort is set by another warp of the block.
__device__ __forceinline__ bool mbarWaitBounded(uint32_t bar, uint32_t parity, const volatile int* abort = nullptr) {
  if (mbarTryWait(bar, parity)) return true;
  const uint64_t t0 = globalTimerNs();
  for (long long it = 0; it < kWaitLimit; ++it) {
    if (mbarTryWaitSleep(bar, parity, 20000)) return true;
    if (abort && *abort) return false;
    if (globalTimerNs() - t0 > kWaitNs) return false;
  }
  return false;
}
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Arrival (release semantics, CTA scope) on an mbarrier.
__device__ __forceinline__ void mbarArrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Barrier `id` (1..15) among `count` threads (a multiple of 32) that also
// returns, to every one of them, the OR of their `v`.
__device__ __forceinline__ bool namedBarOr(int id, int count, bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %3, 0;\n\t"
      "bar.red.or.pred p, %1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(out)
      : "r"(id), "r"(count), "r"(static_cast<uint32_t>(v))
      : "memory");
  return out != 0;
}
// Named barrier without a reduction (bar.sync id, count).
__device__ __forceinline__ void namedBarSync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
// Hint: bring [src, src + bytes) into L2 (no completion, no shared memory).
__device__ __forceinline__ void prefetchL2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// The fused prologue (the same functor as Pro<W> in kernels_precond.cu):
// the right-hand side of the substitution, computed per row.
template <class W>
struct SPro {
  int kind;
  const W* __restrict__ b;
  const W* __restrict__ r;
  W* pOrS;
  const W* __restrict__ v;
  const KState* st;
  // Batches: the state of block b is st[stIndex[b]] (null: st itself).
  const int* stIndex = nullptr;
  __device__ __forceinline__ const KState* state() const {
    return st && stIndex ? st + stIndex[blockIdx.x] : st;
  }
  __device__ __forceinline__ W operator()(int i, W beta, W omega, W alpha, bool first) const {
    if (kind == static_cast<int>(Prologue::Plain)) return b[i];
    if (kind == static_cast<int>(Prologue::PUpdate)) {
      W p = first ? r[i] : add(r[i], mul(beta, sub(pOrS[i], mul(omega, v[i]))));
      pOrS[i] = p;
      return p;
    }
    W s = sub(r[i], mul(alpha, v[i]));
    pOrS[i] = s;
    return s;
  }
  // The same for rows i0 + j * stride (j < N, rows below n), all loads
  // issued before any store, so that the N rows' loads overlap.
  template <int N>
  __device__ __forceinline__ void rows(int i0, int stride, int n, W beta, W omega, W alpha, bool first,
                                       W (&out)[N]) const {
    bool in[N];
#pragma unroll
    for (int j = 0; j < N; ++j) in[j] = i0 + j * stride < n;
    if (kind == static_cast<int>(Prologue::Plain)) {
#pragma unroll
      for (int j = 0; j < N; ++j) out[j] = in[j] ? b[i0 + j * stride] : W(0);
      return;
    }
    W rr[N], pp[N], vv[N];
    const bool pu = kind == static_cast<int>(Prologue::PUpdate);
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const int i = i0 + j * stride;
      rr[j] = in[j] ? r[i] : W(0);
      pp[j] = in[j] && pu && !first ? pOrS[i] : W(0);
      vv[j] = in[j] && !(pu && first) ? v[i] : W(0);
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      if (pu) out[j] = first ? rr[j] : add(rr[j], mul(beta, sub(pp[j], mul(omega, vv[j]))));
      else out[j] = sub(rr[j], mul(alpha, vv[j]));
      if (in[j]) pOrS[i0 + j * stride] = out[j];
    }
  }
};


}  // namespace dev
}  // namespace gr

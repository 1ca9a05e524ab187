// Bulk asynchronous copies into shared memory with mbarrier completion
// (cp.async.bulk, no multicast: a block copies only from this GPU's global
// memory into its own shared memory), and the fused PBiCGStab prologue
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
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
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
};


}  // namespace dev
}  // namespace gr

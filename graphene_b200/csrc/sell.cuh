// SELL-32 row kernels shared by the SpMV, residual and fused Krylov kernels.
#pragma once

#include "device.hpp"
#include "devmath.cuh"

namespace gr {
namespace dev {

template <class MV>
struct SellView {
  int n, nChunks;
  const int* __restrict__ base;
  const int2* __restrict__ ent;  // float coefficients: {column, value bits}
  const int* __restrict__ col;   // double coefficients: columns ...
  const MV* __restrict__ val;    // ... and values
  const MV* __restrict__ diag;
};

// Splits one launch into independent systems (a batch of block-diagonal
// systems solved together). Block b belongs to system sys[b] and is number
// rank[b] of that system's blocks; system s owns blocks [block0[s],
// block0[s] + blocks[s]) and rows [row0[s], rowEnd[s]), row0 a multiple of
// 32. Without tables (blockSys null) the whole launch is one system, and the
// kernels behave exactly as before.
struct SegView {
  const int* blockSys = nullptr;
  const int* blockRank = nullptr;
  const int* sysBlocks = nullptr;
  const int* sysBlock0 = nullptr;
  const int* sysRow0 = nullptr;
  const int* sysRowEnd = nullptr;
};

struct SegPos {
  int sys, rank, nb, b0, r0, r1;
};

__device__ __forceinline__ SegPos segPos(const SegView& g, int n) {
  if (!g.blockSys) return {0, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x), 0, 0, n};
  const int s = g.blockSys[blockIdx.x];
  return {s, g.blockRank[blockIdx.x], g.sysBlocks[s], g.sysBlock0[s], g.sysRow0[s], g.sysRowEnd[s]};
}

// Loads x[i] converted to the accumulation type.
template <class Acc, class XT>
__device__ __forceinline__ Acc loadX(const XT* __restrict__ x, int i) {
  return cvt<Acc>(__ldg(x + i));
}

// Row sum of one row of a SELL-32 chunk, in Acc: diag * x[row] first, then
// the off-diagonal products added in stored order (padding slots have
// column -1 and are skipped, so the result is the sequential row sum).
// The loads of up to B entries are issued before the dependent gathers of x
// so that a warp keeps many memory requests in flight; the matrix stream is
// read with evict-first loads so that x stays resident in L2.
template <class Acc, class MV, class XT, int B = 8>
__device__ __forceinline__ Acc sellRowSum(const SellView<MV>& A, const XT* __restrict__ x, int row,
                                          int s0, int K, int lane) {
  Acc acc = mul(cvt<Acc>(__ldg(A.diag + row)), loadX<Acc>(x, row));
  for (int k = 0; k < K; k += B) {
    int c[B];
    MV a[B];
    if constexpr (sizeof(MV) == 4) {
      const int2* p = A.ent + s0 + lane + 32 * k;
#pragma unroll
      for (int j = 0; j < B; ++j) {
        int2 e = (k + j < K) ? __ldcs(p + 32 * j) : make_int2(-1, 0);
        c[j] = e.x;
        a[j] = __int_as_float(e.y);
      }
    } else {
      const int* cp = A.col + s0 + lane + 32 * k;
      const MV* vp = A.val + s0 + lane + 32 * k;
#pragma unroll
      for (int j = 0; j < B; ++j) {
        const bool in = k + j < K;
        c[j] = in ? __ldcs(cp + 32 * j) : -1;
        a[j] = in ? __ldcs(vp + 32 * j) : MV(0);
      }
    }
    Acc xv[B];
#pragma unroll
    for (int j = 0; j < B; ++j) xv[j] = c[j] >= 0 ? loadX<Acc>(x, c[j]) : Acc(0);
#pragma unroll
    for (int j = 0; j < B; ++j)
      if (c[j] >= 0) acc = add(acc, mul(cvt<Acc>(a[j]), xv[j]));
  }
  return acc;
}

template <class T> __device__ __forceinline__ double toDouble(T v) { return static_cast<double>(v); }

// Accumulates one stored residual entry into a norm partial.
__device__ __forceinline__ double normStep(double acc, double r, int kind) {
  if (kind == GR_NORM_L2) return __dadd_rn(acc, __dmul_rn(r, r));
  if (kind == GR_NORM_LINF) return fmax(acc, r);
  return __dadd_rn(acc, r);  // L1: signed sum (dsl/tensor/Tensor.cpp:428-430)
}

__device__ __forceinline__ int normOp(int kind) { return kind == GR_NORM_LINF ? RED_MAX : RED_SUM; }

__device__ __forceinline__ double normFinish(double total, int kind) {
  return kind == GR_NORM_L2 ? sqrt(total) : total;
}

}  // namespace dev

template <class MV>
inline dev::SellView<MV> sellView(const DeviceMatrix& A) {
  return dev::SellView<MV>{A.n, A.sell.nChunks, A.sell.base.as<int>(), A.sell.ent.as<int2>(), A.sell.col.as<int>(),
                           A.sell.val.as<MV>(), A.diag.as<MV>()};
}

inline void checkLaunch(const char* name) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("launch of ") + name + " failed: " + cudaGetErrorString(e));
  noteLaunch();
}


}  // namespace gr

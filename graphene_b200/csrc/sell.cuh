// SELL-32 row kernels shared by the SpMV, residual and fused Krylov kernels.
#pragma once

#include "device.hpp"
#include "devmath.cuh"

namespace gr {
namespace dev {

// 16-bit SELL layout codes (column - row is never 0 for an off-diagonal),
// and the most far columns one chunk may have.
constexpr int kSellPad = 0;
constexpr int kSellFar = -32768;
constexpr int kSellMaxFar = 64;

template <class MV>
struct SellView {
  int n, nChunks;
  const int* __restrict__ base;
  const int2* __restrict__ ent;  // 32-bit layout, float coefficients: {column, value bits}
  const int* __restrict__ col;   // 32-bit layout, double coefficients: columns ...
  const MV* __restrict__ val;    // ... and values; the 16-bit layout's values (both types)
  const MV* __restrict__ diag;
  // 16-bit layout (d16 non-null): column - row per slot (kSellPad: padding,
  // kSellFar: the column is the chunk's next far column), far columns in
  // slot order and the number of far entries before each chunk.
  const short* __restrict__ d16;
  const int* __restrict__ farCol;
  const int* __restrict__ farBase;
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

// The slots of SELL chunk c as one warp walks them, k = 0, 1, ... (all 32
// lanes together: the 16-bit layout, C16, resolves far columns with warp
// votes). Lane l reads the slots of row 32c + l.
template <class MV, bool C16>
struct ChunkWalk {
  int s0, K, lane, row;
  int farRun = 0, farReg = 0, farReg2 = 0;
  bool wide = false;  // more than 32 far columns: the second register too

  __device__ __forceinline__ ChunkWalk(const SellView<MV>& A, int c, int lane_) : lane(lane_) {
    row = c * 32 + lane;
    s0 = __ldg(A.base + c);
    K = (__ldg(A.base + c + 1) - s0) >> 5;
    if constexpr (C16) {
      const int farBase = __ldg(A.farBase + c);
      const int nFar = __ldg(A.farBase + c + 1) - farBase;
      // The chunk's far columns (at most kSellMaxFar = 64, checked on the
      // host) live in two registers of the lanes and are handed out by
      // shuffles.
      if (lane < nFar) farReg = __ldg(A.farCol + farBase + lane);
      wide = nFar > 32;
      if (lane + 32 < nFar) farReg2 = __ldg(A.farCol + farBase + 32 + lane);
    }
  }

  // 16-bit layout: the column of a slot with code d (-1: padding). All 32
  // lanes call it together, for their slots of the same k, in k order.
  __device__ __forceinline__ int column(const SellView<MV>& A, int d) {
    const bool far = d == kSellFar;
    const unsigned vote = __ballot_sync(0xffffffffu, far);
    int fc = 0;
    if (vote) {  // warp-uniform
      const int idx = farRun + __popc(vote & ((1u << lane) - 1u));
      fc = __shfl_sync(0xffffffffu, farReg, idx & 31);
      if (wide) {  // warp-uniform
        const int hi = __shfl_sync(0xffffffffu, farReg2, idx & 31);
        if (idx >= 32) fc = hi;
      }
      farRun += __popc(vote);
    }
    return d == kSellPad ? -1 : (far ? fc : row + d);
  }

  // Columns (-1: padding) and coefficients of slots k .. k+B-1 of this lane's
  // row. The loads of all B slots are issued before any is used.
  template <int B>
  __device__ __forceinline__ void load(const SellView<MV>& A, int k, int (&c)[B], MV (&a)[B]) {
    if constexpr (C16) {
      const short* dp = A.d16 + s0 + lane + 32 * k;
      const MV* vp = A.val + s0 + lane + 32 * k;
      short d[B];
#pragma unroll
      for (int j = 0; j < B; ++j) {
        const bool in = k + j < K;
        d[j] = in ? __ldcs(dp + 32 * j) : static_cast<short>(kSellPad);
        a[j] = in ? __ldcs(vp + 32 * j) : MV(0);
      }
#pragma unroll
      for (int j = 0; j < B; ++j) c[j] = column(A, d[j]);
    } else if constexpr (sizeof(MV) == 4) {
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
  }
};

// Row sum of row 32c + lane of SELL chunk c, in Acc: diag * x[row] first,
// then the off-diagonal products added in stored order (padding slots are
// skipped, so the result is the sequential row sum). All 32 lanes of the
// warp call it together; a lane whose row is not `live` (past the matrix or
// the system) returns 0 and touches neither the diagonal nor x. The loads
// of up to B entries are issued before the dependent gathers of x so that a
// warp keeps many memory requests in flight; the matrix stream is read with
// evict-first loads so that x stays resident in L2.
template <class Acc, class MV, class XT, bool C16, int B = C16 ? 4 : 8>
__device__ __forceinline__ Acc sellRowSum(const SellView<MV>& A, const XT* __restrict__ x, int c, int lane,
                                          bool live) {
  ChunkWalk<MV, C16> w(A, c, lane);
  const int row = w.row;
  Acc acc = live ? mul(cvt<Acc>(__ldg(A.diag + row)), loadX<Acc>(x, row)) : Acc(0);
  for (int k = 0; k < w.K; k += B) {
    MV a[B];
    int cl[B];
    w.template load<B>(A, k, cl, a);
    Acc xv[B];
#pragma unroll
    for (int j = 0; j < B; ++j) xv[j] = cl[j] >= 0 ? loadX<Acc>(x, cl[j]) : Acc(0);
#pragma unroll
    for (int j = 0; j < B; ++j)
      if (cl[j] >= 0) acc = add(acc, mul(cvt<Acc>(a[j]), xv[j]));
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
  return dev::SellView<MV>{A.n,
                           A.sell.nChunks,
                           A.sell.base.as<int>(),
                           A.sell.compact ? nullptr : A.sell.ent.as<int2>(),
                           A.sell.compact ? nullptr : A.sell.col.as<int>(),
                           A.sell.val.as<MV>(),
                           A.diag.as<MV>(),
                           A.sell.compact ? A.sell.d16.as<short>() : nullptr,
                           A.sell.farCol.as<int>(),
                           A.sell.farBase.as<int>()};
}

inline void checkLaunch(const char* name) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("launch of ") + name + " failed: " + cudaGetErrorString(e));
  noteLaunch();
}


}  // namespace gr

// Device arithmetic helpers: IEEE operations with no contraction, the
// double-word ("twofloat") algorithms, and deterministic block/grid
// reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gr {
namespace dev {

// Every arithmetic step of the hot path is written as one rounded IEEE
// operation so that results do not depend on whether the compiler would
// fuse a multiply and an add. The CPU oracle is compiled the same way.
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

template <class T> __device__ __forceinline__ T cvt(float v);
template <class T> __device__ __forceinline__ T cvt(double v);
template <> __device__ __forceinline__ float cvt<float>(float v) { return v; }
template <> __device__ __forceinline__ float cvt<float>(double v) { return __double2float_rn(v); }
template <> __device__ __forceinline__ double cvt<double>(float v) { return static_cast<double>(v); }
template <> __device__ __forceinline__ double cvt<double>(double v) { return v; }

// ---- double-word arithmetic ------------------------------------------
// A value x = h + l with |l| <= ulp(h)/2, two floats. Algorithms from
// M. Joldes, J.-M. Muller, V. Popescu, "Tight and rigorous error bounds for
// basic building blocks of double-word arithmetic", ACM TOMS 44(2), 2017:
// 2Sum, Fast2Sum, 2Prod (with FMA), DWPlusFP (Alg. 4), AccurateDWPlusDW
// (Alg. 6) and DWTimesFP with FMA (Alg. 9 in that paper's numbering of the
// FMA variants).
struct dw {
  float h, l;
};

__device__ __forceinline__ dw twoSum(float a, float b) {
  float s = __fadd_rn(a, b);
  float ap = __fsub_rn(s, b);
  float bp = __fsub_rn(s, ap);
  float da = __fsub_rn(a, ap);
  float db = __fsub_rn(b, bp);
  return {s, __fadd_rn(da, db)};
}
__device__ __forceinline__ dw fastTwoSum(float a, float b) {
  float s = __fadd_rn(a, b);
  float z = __fsub_rn(s, a);
  return {s, __fsub_rn(b, z)};
}
__device__ __forceinline__ dw twoProd(float a, float b) {
  float p = __fmul_rn(a, b);
  return {p, __fmaf_rn(a, b, -p)};
}
__device__ __forceinline__ dw dwPlusFp(dw x, float y) {
  dw s = twoSum(x.h, y);
  float v = __fadd_rn(x.l, s.l);
  return fastTwoSum(s.h, v);
}
__device__ __forceinline__ dw dwPlusDw(dw x, dw y) {
  dw s = twoSum(x.h, y.h);
  dw t = twoSum(x.l, y.l);
  float c = __fadd_rn(s.l, t.h);
  dw v = fastTwoSum(s.h, c);
  float w = __fadd_rn(t.l, v.l);
  return fastTwoSum(v.h, w);
}
__device__ __forceinline__ dw dwTimesFp(dw x, float y) {
  dw c = twoProd(x.h, y);
  float cl3 = __fmaf_rn(x.l, y, c.l);
  return fastTwoSum(c.h, cl3);
}
__device__ __forceinline__ dw dwNeg(dw x) { return {-x.h, -x.l}; }
__device__ __forceinline__ float dwToFloat(dw x) { return __fadd_rn(x.h, x.l); }

// ---- reductions --------------------------------------------------------
// Deterministic FP64 reductions: each thread accumulates its elements in a
// fixed order, a block reduces with a fixed shuffle/shared-memory tree, and
// the last block to finish reduces the per-block partials in block order.
// Results depend only on the launch geometry, which is fixed per matrix.

enum RedOp : int { RED_SUM = 0, RED_MAX = 1 };

__device__ __forceinline__ double redCombine(double a, double b, int op) {
  return op == RED_MAX ? fmax(a, b) : __dadd_rn(a, b);
}

__device__ __forceinline__ double redIdentity(int op) { return op == RED_MAX ? -INFINITY : 0.0; }

// Reduces NV values across the block; the result is valid in thread 0.
// smem must hold 32 * NV doubles.
template <int NV>
__device__ __forceinline__ void blockReduce(double (&v)[NV], const int (&ops)[NV], double* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[j] = redCombine(v[j], __shfl_down_sync(0xffffffffu, v[j], o), ops[j]);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) smem[warp * NV + j] = v[j];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      v[j] = lane < nw ? smem[lane * NV + j] : redIdentity(ops[j]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[j] = redCombine(v[j], __shfl_down_sync(0xffffffffu, v[j], o), ops[j]);
    }
  }
}

// Completes a grid reduction over `nb` blocks, this block being number
// `rank` of them. Every block calls this with its block-reduced values (valid
// in thread 0). Returns true in exactly one block (the last to arrive); in
// that block, thread 0's out[] holds the totals, combined in rank order. The
// counter is reset for the next launch.
template <int NV>
__device__ __forceinline__ bool gridReduceRank(double (&v)[NV], const int (&ops)[NV], double* partials,
                                               unsigned* counter, double* smem, double (&out)[NV], int rank,
                                               int nb) {
  __shared__ bool amLast;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) partials[rank * NV + j] = v[j];
    __threadfence();
    unsigned ticket = atomicAdd(counter, 1u);
    amLast = (ticket == static_cast<unsigned>(nb) - 1);
  }
  __syncthreads();
  if (!amLast) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = redIdentity(ops[j]);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = redCombine(acc[j], __ldcg(partials + b * NV + j), ops[j]);
  }
  blockReduce<NV>(acc, ops, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = acc[j];
    *counter = 0u;
    __threadfence();
  }
  return true;
}

// Grid reduction over the whole launch (block rank = blockIdx.x).
template <int NV>
__device__ __forceinline__ bool gridReduce(double (&v)[NV], const int (&ops)[NV], double* partials,
                                           unsigned* counter, double* smem, double (&out)[NV]) {
  return gridReduceRank<NV>(v, ops, partials, counter, smem, out, static_cast<int>(blockIdx.x),
                            static_cast<int>(gridDim.x));
}

}  // namespace dev
}  // namespace gr

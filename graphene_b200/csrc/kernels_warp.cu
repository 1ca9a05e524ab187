// Warp-per-tile block-ILU(0) / DILU substitution.
//
// Same arithmetic as iluApplyKernel (ilu/Solver.cpp:367-550, level by
// level), organised for latency: one warp owns one tile, so a level ends
// with __syncwarp() instead of a block barrier, and the shared memory of a
// block is only the tile's slice of x plus its level table, so many tiles
// are resident per SM. Each lane keeps the entries of its rows of the next
// two levels in registers (coalesced read-only loads issued two levels
// ahead), so a level's work waits on shared memory only. Rows beyond
// 32*J per level and entries beyond EM per row are read directly.
//
// Input: the tile byte stream and level table of SweepStream (device.hpp).
#include <algorithm>

#include "devmath.cuh"
#include "krylov.hpp"
#include "sell.cuh"

namespace gr {
namespace dev {

template <class W>
struct WPro {
  int kind;
  const W* __restrict__ b;
  const W* __restrict__ r;
  W* pOrS;
  const W* __restrict__ v;
  const KState* st;
  __device__ __forceinline__ W operator()(int i, W beta, W omega, W alpha, bool first) const {
    if (kind == static_cast<int>(Prologue::Plain)) return b[i];
    if (kind == static_cast<int>(Prologue::PUpdate)) {
      // pA = rA + beta * (pA - omega * AyA) (pbicgstab/Solver.cpp:98-101)
      W p = first ? r[i] : add(r[i], mul(beta, sub(pOrS[i], mul(omega, v[i]))));
      pOrS[i] = p;
      return p;
    }
    // sA = rA - alpha * AyA (pbicgstab/Solver.cpp:129)
    W s = sub(r[i], mul(alpha, v[i]));
    pOrS[i] = s;
    return s;
  }
};

__device__ __forceinline__ uint32_t p16(uint32_t b) { return (b + 15u) & ~15u; }

template <class MV, int J, int EM>
struct Stage {
  int il[J];
  MV iv[J];
  int c[J][EM];
  MV v[J][EM];
};

// Segment pointers of one level (see SweepStream's stream layout).
template <class MV>
struct LevelPtr {
  const int* rows;
  const MV* inv;
  const int* cols;
  const MV* vals;
  int k, E;
  bool hasInv;
  __device__ __forceinline__ LevelPtr(const unsigned char* g, int4 d) {
    k = d.y;
    E = d.z;
    hasInv = d.w != 0;
    const unsigned char* p = g + d.x + 16;
    rows = reinterpret_cast<const int*>(p);
    p += p16(4u * k);
    inv = reinterpret_cast<const MV*>(p);
    if (hasInv) p += p16(static_cast<uint32_t>(sizeof(MV)) * k);
    cols = reinterpret_cast<const int*>(p);
    p += p16(4u * E * k);
    vals = reinterpret_cast<const MV*>(p);
  }
};

template <class MV, int J, int EM>
__device__ __forceinline__ void prefetch(Stage<MV, J, EM>& s, const unsigned char* g, const int4* tab, int L,
                                         int nLev, int lane) {
  if (L >= nLev) return;
  const LevelPtr<MV> lp(g, tab[L]);
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int r = j * 32 + lane;
    const bool in = r < lp.k;
    s.il[j] = in ? __ldg(lp.rows + r) : 0;
    s.iv[j] = (in && lp.hasInv) ? __ldg(lp.inv + r) : MV(0);
#pragma unroll
    for (int e = 0; e < EM; ++e) {
      const bool ine = in && e < lp.E;
      s.c[j][e] = ine ? __ldg(lp.cols + e * lp.k + r) : -1;
      s.v[j][e] = ine ? __ldg(lp.vals + e * lp.k + r) : MV(0);
    }
  }
}

// Finishes row il given the accumulated temp (forward or backward step).
template <class W>
__device__ __forceinline__ void finishRow(W* xs, int il, W temp, W iv, bool upper, bool dilu) {
  if (!upper) xs[il] = dilu ? mul(temp, iv) : temp;
  else xs[il] = dilu ? add(xs[il], mul(temp, iv)) : mul(add(xs[il], temp), iv);
}

template <class MV, class W, int J, int EM>
__device__ __forceinline__ void process(const Stage<MV, J, EM>& s, const unsigned char* g, const int4* tab, int L,
                                        bool upper, bool dilu, W* xs, int lane) {
  const LevelPtr<MV> lp(g, tab[L]);
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int r = j * 32 + lane;
    if (r < lp.k) {
      const int il = s.il[j];
      W temp = upper ? W(0) : xs[il];
      W xv[EM];
#pragma unroll
      for (int e = 0; e < EM; ++e) xv[e] = s.c[j][e] >= 0 ? xs[s.c[j][e]] : W(0);
#pragma unroll
      for (int e = 0; e < EM; ++e)
        if (s.c[j][e] >= 0) temp = sub(temp, mul(cvt<W>(s.v[j][e]), xv[e]));
      for (int e = EM; e < lp.E; ++e) {
        const int c = __ldg(lp.cols + e * lp.k + r);
        if (c < 0) break;
        temp = sub(temp, mul(cvt<W>(__ldg(lp.vals + e * lp.k + r)), xs[c]));
      }
      finishRow(xs, il, temp, cvt<W>(s.iv[j]), upper, dilu);
    }
  }
  // Rows beyond the prefetched ones.
  for (int r = J * 32 + lane; r < lp.k; r += 32) {
    const int il = __ldg(lp.rows + r);
    W temp = upper ? W(0) : xs[il];
    for (int e = 0; e < lp.E; ++e) {
      const int c = __ldg(lp.cols + e * lp.k + r);
      if (c < 0) break;
      temp = sub(temp, mul(cvt<W>(__ldg(lp.vals + e * lp.k + r)), xs[c]));
    }
    finishRow(xs, il, temp, lp.hasInv ? cvt<W>(__ldg(lp.inv + r)) : W(0), upper, dilu);
  }
}

template <class MV, class W, int J, int EM>
__global__ void __launch_bounds__(32) iluWarpKernel(const unsigned char* __restrict__ stream,
                                                     const long long* __restrict__ tileOffset,
                                                     const int4* __restrict__ levelTable,
                                                     const int* __restrict__ tileLevel,
                                                     const int* __restrict__ tileStart, int tableSlots, bool dilu,
                                                     WPro<W> pro, W* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (pro.st && pro.st->done) return;
  const int T = blockIdx.x;
  const int lane = threadIdx.x;
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  const int lv0 = tileLevel[T];
  const int nLev = tileLevel[T + 1] - lv0;
  const unsigned char* g = stream + tileOffset[T];
  const int nL = __ldg(reinterpret_cast<const int*>(g));
  int4* tab = reinterpret_cast<int4*>(smem);
  W* xs = reinterpret_cast<W*>(smem + 16 * static_cast<size_t>(tableSlots));
  for (int i = lane; i < nLev; i += 32) tab[i] = levelTable[lv0 + i];
  {
    W beta = W(0), omega = W(0), alpha = W(0);
    bool first = true;
    if (pro.st) {
      beta = cvt<W>(pro.st->beta);
      omega = cvt<W>(pro.st->omega);
      alpha = cvt<W>(pro.st->alpha);
      first = pro.st->iter == 0;
    }
    for (int i = lane; i < nRows; i += 32) xs[i] = pro(base + i, beta, omega, alpha, first);
  }
  __syncwarp();
  Stage<MV, J, EM> s0, s1;
  prefetch(s0, g, tab, 0, nLev, lane);
  prefetch(s1, g, tab, 1, nLev, lane);
  for (int L = 0; L < nLev; L += 2) {
    process<MV, W, J, EM>(s0, g, tab, L, L >= nL, dilu, xs, lane);
    __syncwarp();
    prefetch(s0, g, tab, L + 2, nLev, lane);
    if (L + 1 < nLev) {
      process<MV, W, J, EM>(s1, g, tab, L + 1, L + 1 >= nL, dilu, xs, lane);
      __syncwarp();
      prefetch(s1, g, tab, L + 3, nLev, lane);
    }
  }
  for (int i = lane; i < nRows; i += 32) y[base + i] = xs[i];
}

}  // namespace dev

// ---------------------------------------------------------------------------
namespace {

template <class MV, class W, int J>
void warpApplyT(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu, const PrologueArgs& p, void* y,
                cudaStream_t s) {
  const size_t smem = 16 * static_cast<size_t>(S.maxTileLevels) + A.host->maxTileRows * sizeof(W);
  auto kernel = dev::iluWarpKernel<MV, W, J, 4>;
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
  dev::WPro<W> pro{static_cast<int>(p.kind), static_cast<const W*>(p.b), static_cast<const W*>(p.r),
                   static_cast<W*>(p.pOrS), static_cast<const W*>(p.v), p.st};
  kernel<<<A.P, 32, smem, s>>>(static_cast<const unsigned char*>(stream), S.tileOffset.as<long long>(),
                               S.levelTable.as<int4>(), S.tileLevel.as<int>(), A.tileStart.as<int>(),
                               S.maxTileLevels, dilu, pro, static_cast<W*>(y));
  checkLaunch("ilu_warp");
}

template <class MV, class W>
void warpApplyJ(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu, const PrologueArgs& p, void* y,
                int J, cudaStream_t s) {
  if (J <= 1) warpApplyT<MV, W, 1>(A, S, stream, dilu, p, y, s);
  else if (J == 2) warpApplyT<MV, W, 2>(A, S, stream, dilu, p, y, s);
  else warpApplyT<MV, W, 4>(A, S, stream, dilu, p, y, s);
}

}  // namespace

int iluWarpRowsPerLane(const DeviceMatrix& A, const SweepStream& S) {
  // Every row appears in one forward and one backward level.
  const double avg = 2.0 * A.n / std::max<i64>(1, S.numLevels);
  return avg <= 24 ? 1 : (avg <= 56 ? 2 : 4);
}

size_t iluWarpSmem(const DeviceMatrix& A, const SweepStream& S, DType W) {
  return 16 * static_cast<size_t>(S.maxTileLevels) + A.host->maxTileRows * dtypeSize(W);
}

void launchIluWarp(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu, const PrologueArgs& pro,
                   void* y, DType W, int J, cudaStream_t s) {
  if (A.vt == DType::F32 && W == DType::F32) warpApplyJ<float, float>(A, S, stream, dilu, pro, y, J, s);
  else if (A.vt == DType::F32 && W == DType::F64) warpApplyJ<float, double>(A, S, stream, dilu, pro, y, J, s);
  else if (A.vt == DType::F64 && W == DType::F64) warpApplyJ<double, double>(A, S, stream, dilu, pro, y, J, s);
  else fail(GR_EUNSUPPORTED, "ILU with float64 coefficients needs float64 vectors");
}

}  // namespace gr

// Block-ILU(0) / DILU substitution through a host-scheduled shared-memory
// ring (ilu/Solver.cpp:367-550, level by level; same arithmetic and order as
// the other substitution kernels).
//
// One thread block per group of consecutive tiles, run in lockstep (level l
// of the block is level l of each of its tiles). The level blocks (LevelRing, device.hpp)
// are copied from global memory into a shared-memory ring with one bulk
// asynchronous copy per level (cp.async.bulk, completion on one of
// kRingBarriers mbarriers; no multicast: a block copies only its own tile's
// bytes from this GPU's memory). The host fixed each level's ring offset and
// the level after which its copy is issued, so the kernel does no ring
// arithmetic: a level's rows, inverse diagonal and (column, value) entries
// sit at fixed offsets. Per level: four compute warps compute the level's
// rows from shared memory, one producer warp issues the copies that the
// previous level released and another waits until the next level has
// landed; one barrier ends the level.
//
// Every wait is bounded; when one runs out the block records GR_ETIMEOUT in
// the matrix's error word, stops at the next barrier, and the issuing lane
// waits (bounded) for the copies still in flight before the block exits.
#include <algorithm>

#include "bulk.cuh"
#include "device.hpp"
#include "devmath.cuh"
#include "krylov.hpp"
#include "sell.cuh"

namespace gr {
namespace dev {

// Four compute warps, an issuing warp and a waiting warp per block.
constexpr int kRingCompute = 128;
constexpr int kRingThreads = kRingCompute + 64;
constexpr int kPrefetchAhead = 0;  // default bytes kept prefetched into L2 beyond the issued copies

// Entry of a level block: column and value (the value at byte 4 for float,
// byte 8 for double).
template <class MV>
__device__ __forceinline__ void loadEntry(const unsigned char* p, int& c, MV& v);
template <>
__device__ __forceinline__ void loadEntry<float>(const unsigned char* p, int& c, float& v) {
  const int2 e = *reinterpret_cast<const int2*>(p);
  c = e.x;
  v = __int_as_float(e.y);
}
template <>
__device__ __forceinline__ void loadEntry<double>(const unsigned char* p, int& c, double& v) {
  const int4 e = *reinterpret_cast<const int4*>(p);
  c = e.x;
  v = __hiloint2double(e.w, e.z);
}

__device__ __forceinline__ bool waitBar(uint32_t bar, uint32_t parity) {
  for (long long it = 0; it < kWaitLimit; ++it)
    if (mbarTryWait(bar, parity)) return true;
  return false;
}

// temp -= sum_e value_e * xs[column_e] over a row's E entries in order.
// Padding entries (column = the zero slot, value 0) leave temp unchanged.
// Rows of up to four entries load all their entries, then all x values,
// before the arithmetic.
template <class MV, bool UNROLL, class W>
__device__ __forceinline__ W ringRowDot(W temp, const unsigned char* p, uint32_t stride, int E, int zeroSlot,
                                        const W* xs) {
  constexpr uint32_t kEnt = sizeof(MV) == 4 ? 8 : 16;
  (void)kEnt;
  if (UNROLL && E <= 4) {
    int c[4];
    MV v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (e < E) {
        loadEntry<MV>(p + e * stride, c[e], v[e]);
      } else {
        c[e] = zeroSlot;
        v[e] = MV(0);
      }
    }
    W xv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) xv[e] = xs[c[e]];
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (e < E) temp = sub(temp, mul(cvt<W>(v[e]), xv[e]));
    return temp;
  }
  for (int e = 0; e < E; ++e, p += stride) {
    int c;
    MV v;
    loadEntry<MV>(p, c, v);
    temp = sub(temp, mul(cvt<W>(v), xs[c]));
  }
  return temp;
}

template <class MV, class W, bool UNROLL>
__global__ void __launch_bounds__(kRingThreads) iluRingKernel(const unsigned char* __restrict__ stream,
                                                               const long long* __restrict__ tileOffset,
                                                               const int4* __restrict__ meta,
                                                               const int* __restrict__ tileLevel,
                                                               const int* __restrict__ blockStart, int ringBytes,
                                                               int metaLevels, uint32_t l2Ahead, bool dilu,
                                                               SPro<W> pro, W* __restrict__ y, int* errFlag) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int abortFlag;
  const KState* st = pro.state();
  if (st && st->done) return;
  constexpr uint32_t kEnt = sizeof(MV) == 4 ? 8 : 16;
  const int T = blockIdx.x;
  const int base = blockStart[T];
  const int nRows = blockStart[T + 1] - base;
  const int lv0 = tileLevel[T];
  const int L = tileLevel[T + 1] - lv0;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);  // kRingBarriers level barriers + 1 for the table
  int4* mt = reinterpret_cast<int4*>(smem + 256);
  unsigned char* ring = smem + 256 + 32 * metaLevels;
  W* xs = reinterpret_cast<W*>(ring + ringBytes);
  const unsigned char* g = stream + tileOffset[T];
  const bool producer = threadIdx.x >= kRingCompute;     // the two producer warps
  const bool lead = threadIdx.x == kRingCompute;         // issues the copies
  const bool waiter = threadIdx.x == kRingCompute + 32;  // waits for the next level

  if (lead) {
    abortFlag = 0;
    for (int i = 0; i <= kRingBarriers; ++i) mbarInit(smemAddr(bars + i), 1);
    fenceBarrierInit();
    const uint32_t tb = static_cast<uint32_t>(L) * 32u;
    mbarExpectTx(smemAddr(bars + kRingBarriers), tb);
    bulkLoad(smemAddr(mt), meta + 2 * static_cast<size_t>(lv0), tb, smemAddr(bars + kRingBarriers));
  }
  // Prologue into the tile's slice of x while the level table lands; the
  // slot after the slice is the zero that padding entries read.
  {
    W beta = W(0), omega = W(0), alpha = W(0);
    bool first = true;
    if (st) {
      beta = cvt<W>(st->beta);
      omega = cvt<W>(st->omega);
      alpha = cvt<W>(st->alpha);
      first = st->iter == 0;
    }
    for (int i = threadIdx.x; i < nRows; i += blockDim.x) xs[i] = pro(base + i, beta, omega, alpha, first);
    if (lead) xs[nRows] = W(0);
  }
  // The issuing lane copies levels in order: `next` is the next level to
  // copy (its table entries held in na / nia), `src` its byte offset in the
  // block's stream, `pf` the L2 prefetch frontier.
  int next = 0, nia = 0;
  int4 na = make_int4(0, 0, 0, 0);
  uint32_t src = 0, pf = 0;
  const uint32_t tileBytes = static_cast<uint32_t>(tileOffset[T + 1] - tileOffset[T]);
  auto issueUpTo = [&](int consumed) {
    while (next < L && nia <= consumed) {
      const uint32_t bar = smemAddr(bars + (next % kRingBarriers));
      mbarExpectTx(bar, static_cast<uint32_t>(na.z));
      bulkLoad(smemAddr(ring + na.w), g + src, static_cast<uint32_t>(na.z), bar);
      src += static_cast<uint32_t>(na.z);
      if (++next < L) {
        na = mt[2 * next];
        nia = mt[2 * next + 1].z;
      }
    }
    if (pf < src) pf = src;
    const uint32_t until = min(tileBytes, src + l2Ahead);
    if (pf < until) {
      prefetchL2(g + pf, until - pf);
      pf = until;
    }
  };
  bool tableLanded = false;
  if (lead) {
    if (!waitBar(smemAddr(bars + kRingBarriers), 0)) {
      abortFlag = 1;
    } else {
      tableLanded = true;
      na = mt[0];
      nia = mt[1].z;
      issueUpTo(-1);
      if (L > 0 && !waitBar(smemAddr(bars), 0)) abortFlag = 1;
    }
  }
  __syncthreads();
  int consumed = -1;  // last level every thread finished
  if (!abortFlag) {
    for (int l = 0; l < L; ++l) {
      if (producer) {
        // Copies released by level l - 1 (finished by every thread before
        // the previous barrier); meanwhile the waiting warp waits until level
        // l + 1 has landed.
        if (lead && l > 0 && next < L) {
          fenceProxyAsync();
          issueUpTo(l - 1);
        }
        if (waiter && l + 1 < L &&
            !waitBar(smemAddr(bars + ((l + 1) % kRingBarriers)), ((l + 1) / kRingBarriers) & 1))
          abortFlag = 1;
      } else {
        const int4 a = mt[2 * l], b = mt[2 * l + 1];
        const int k = a.x, E = a.y;
        const unsigned char* blk = ring + a.w;
        const int* rows = reinterpret_cast<const int*>(blk);
        const MV* inv = reinterpret_cast<const MV*>(blk + b.x);
        const unsigned char* ents = blk + b.y;
        const uint32_t stride = kEnt * static_cast<uint32_t>(k);
        if (!b.w) {
          // Forward substitution (ilu/Solver.cpp:380-411).
          for (int q = threadIdx.x; q < k; q += kRingCompute) {
            const int il = rows[q];
            const W temp = ringRowDot<MV, UNROLL>(xs[il], ents + kEnt * q, stride, E, nRows, xs);
            xs[il] = dilu ? mul(temp, cvt<W>(inv[q])) : temp;
          }
        } else {
          // Backward substitution (ilu/Solver.cpp:413-442).
          for (int q = threadIdx.x; q < k; q += kRingCompute) {
            const int il = rows[q];
            const W temp = ringRowDot<MV, UNROLL>(W(0), ents + kEnt * q, stride, E, nRows, xs);
            const W iv = cvt<W>(inv[q]);
            xs[il] = dilu ? add(xs[il], mul(temp, iv)) : mul(add(xs[il], temp), iv);
          }
        }
      }
      __syncthreads();
      consumed = l;
      if (abortFlag) break;
    }
  }
  if (abortFlag) {
    if (lead) {
      atomicExch(errFlag, GR_ETIMEOUT);
      // Let the copies already issued land before the block's shared memory
      // is released (bounded).
      if (!tableLanded) waitBar(smemAddr(bars + kRingBarriers), 0);
      for (int j = consumed + 1; j < next; ++j) waitBar(smemAddr(bars + (j % kRingBarriers)), (j / kRingBarriers) & 1);
    }
    return;
  }
  for (int i = threadIdx.x; i < nRows; i += blockDim.x) y[base + i] = xs[i];
}

}  // namespace dev

// ---------------------------------------------------------------------------
size_t iluRingSmem(const DeviceMatrix& A, const LevelRing& R, DType W) {
  (void)A;
  return 256 + 32 * static_cast<size_t>(R.maxTileLevels) + static_cast<size_t>(R.ringBytes) +
         static_cast<size_t>(R.maxGroupRows + 1) * dtypeSize(W);
}

void launchRingPack(DeviceMatrix& A, const LevelRing& R, void* stream, const void* F, const void* inv,
                    cudaStream_t s) {
  launchPackBytes(A, R.templ.get(), R.bytes, R.valPos.as<int>(), R.valSrc.as<int>(), R.nVal, R.invPos.as<int>(),
                  R.invSrc.as<int>(), R.nInv, stream, F, inv, s);
}

namespace {
template <class MV, class W>
void ringApplyT(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& p, void* y,
                int l2Ahead, bool unroll, cudaStream_t s) {
  const size_t smem = iluRingSmem(A, R, dtypeOf<W>());
  auto kernel = unroll ? dev::iluRingKernel<MV, W, true> : dev::iluRingKernel<MV, W, false>;
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
  if (p.stIndex && R.group != 1) fail(GR_EUNSUPPORTED, "batched solves run one tile per block");
  dev::SPro<W> pro{static_cast<int>(p.kind), static_cast<const W*>(p.b), static_cast<const W*>(p.r),
                   static_cast<W*>(p.pOrS), static_cast<const W*>(p.v), p.st, p.stIndex};
  kernel<<<R.numGroups, dev::kRingThreads, smem, s>>>(static_cast<const unsigned char*>(stream),
                                             R.tileOffset.as<long long>(), R.meta.as<int4>(), R.tileLevel.as<int>(),
                                             R.groupStart.as<int>(),
                                             static_cast<int>(R.ringBytes), R.maxTileLevels,
                                             static_cast<uint32_t>(l2Ahead < 0 ? dev::kPrefetchAhead : l2Ahead) & ~15u, dilu, pro,
                                             static_cast<W*>(y), A.errFlag.as<int>());
  checkLaunch("ilu_ring");
}
}  // namespace

void launchIluRing(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& pro,
                   void* y, DType W, int l2Ahead, bool unroll, cudaStream_t s) {
  if (A.vt == DType::F32 && W == DType::F32) ringApplyT<float, float>(A, R, stream, dilu, pro, y, l2Ahead, unroll, s);
  else if (A.vt == DType::F32 && W == DType::F64)
    ringApplyT<float, double>(A, R, stream, dilu, pro, y, l2Ahead, unroll, s);
  else if (A.vt == DType::F64 && W == DType::F64)
    ringApplyT<double, double>(A, R, stream, dilu, pro, y, l2Ahead, unroll, s);
  else fail(GR_EUNSUPPORTED, "ILU apply with float64 coefficients and float32 vectors");
}

}  // namespace gr

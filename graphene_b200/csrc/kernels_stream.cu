// Streamed block-ILU(0) / DILU substitution.
//
// Same arithmetic as iluApplyKernel (ilu/Solver.cpp:367-550, level-scheduled)
// but every level's data (row ids, inverse diagonal, columns, factor values)
// comes from a per-tile byte stream (SweepStream) that is copied into a
// shared-memory ring buffer with bulk asynchronous copies
// (cp.async.bulk, completion tracked by one mbarrier per ring chunk). One
// elected thread keeps up to kRingChunks chunks in flight ahead of the level
// being processed, so a level's work reads only shared memory and the
// per-level cost is a barrier instead of an HBM round trip. Every copy is a
// single-CTA bulk copy of the block's own tile bytes from this GPU's memory.
//
// Every wait on an mbarrier is bounded; a wait that runs out sets the
// matrix's error word to GR_ETIMEOUT, all threads leave the level loop
// together at the next barrier, and the elected thread waits (bounded) for
// its outstanding copies before the block exits.
#include <algorithm>

#include "bulk.cuh"
#include "devmath.cuh"
#include "krylov.hpp"
#include "sell.cuh"

namespace gr {
namespace dev {

constexpr int kRingChunks = 8;

// Default number of chunks beyond the ring that the producer keeps
// prefetched into L2, so that a refill reads L2 instead of HBM.
constexpr int kPrefetchChunks = 2 * kRingChunks;

// temp -= sum_e val_e * xs[col_e] over a row's E entries (entry-major, column
// -1 = padding, which only trails a row's entries and carries value 0).
// Rows of up to four entries load all columns and values at once.
template <class MV, bool UNROLL, class W, class RI, class RV>
__device__ __forceinline__ W rowDot(W temp, int E, uint32_t co, uint32_t vo, uint32_t colStride,
                                    uint32_t valStride, const W* xs, RI rdInt, RV rdVal) {
  if (UNROLL && E <= 4) {
    int c[4];
    MV v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      c[e] = e < E ? rdInt(co + e * colStride) : -1;
      v[e] = e < E ? rdVal(vo + e * valStride) : MV(0);
    }
    W xv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) xv[e] = c[e] >= 0 ? xs[c[e]] : W(0);
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (c[e] >= 0) temp = sub(temp, mul(cvt<W>(v[e]), xv[e]));
    return temp;
  }
  for (int e = 0; e < E; ++e, co += colStride, vo += valStride) {
    const int c = rdInt(co);
    if (c < 0) break;
    temp = sub(temp, mul(cvt<W>(rdVal(vo)), xs[c]));
  }
  return temp;
}

__device__ __forceinline__ long long pad16(long long b) { return (b + 15) & ~15ll; }

// Four compute warps and one producer warp per tile.
constexpr int kComputeThreads = 128;
constexpr int kStreamThreads = kComputeThreads + 32;

__device__ __forceinline__ uint32_t pad16u(uint32_t b) { return (b + 15u) & ~15u; }

// One thread block per tile. Per level: the compute warps compute their rows
// from shared memory while the producer warp refills the ring slots of
// chunks that lie wholly before the current level (consumed by earlier
// levels, which every thread finished before the previous barrier) and waits
// until the next level's bytes have landed; one barrier ends the level. The
// ring therefore has to hold two consecutive levels (the host sizes it from
// the largest two-level span, see ringLog2ForLevel).
template <class MV, class W, bool UNROLL>
__global__ void __launch_bounds__(kStreamThreads) iluStreamKernel(const unsigned char* __restrict__ stream,
                                                                   const long long* __restrict__ tileOffset,
                                                                   const int* __restrict__ tileStart, int ringLog2,
                                                                   int prefetchChunks, bool dilu, SPro<W> pro,
                                                                   W* __restrict__ y, int* errFlag) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int abortFlag;
  if (pro.st && pro.st->done) return;
  const int T = blockIdx.x;
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  const long long g0 = tileOffset[T];
  const uint32_t len = static_cast<uint32_t>(tileOffset[T + 1] - g0);
  const uint32_t ringBytes = 1u << ringLog2;
  const uint32_t mask = ringBytes - 1;
  const uint32_t C = ringBytes / kRingChunks;
  const int total = static_cast<int>((len + C - 1) / C);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* ring = smem + 128;
  W* xs = reinterpret_cast<W*>(smem + 128 + ringBytes);
  const unsigned char* g = stream + g0;
  const bool waiter = threadIdx.x >= kComputeThreads;      // the producer warp
  const bool producer = threadIdx.x == kComputeThreads;    // its lane 0 issues copies
  const bool computer = threadIdx.x < kComputeThreads;

  int next = 0;  // next chunk to copy (producer lane)
  auto issue = [&](int c) {
    const uint32_t bytes = min(C, len - static_cast<uint32_t>(c) * C);
    const uint32_t bar = smemAddr(bars + (c % kRingChunks));
    mbarExpectTx(bar, bytes);
    bulkLoad(smemAddr(ring + (c % kRingChunks) * C), g + static_cast<size_t>(c) * C, bytes, bar);
  };
  if (producer) {
    abortFlag = 0;
    for (int r = 0; r < kRingChunks; ++r) mbarInit(smemAddr(bars + r), 1);
    fenceBarrierInit();
  }
  __syncthreads();
  int pf = 0;  // next chunk to prefetch into L2 (producer lane)
  auto prefetchTo = [&](int limit) {
    for (; pf < total && pf < limit; ++pf)
      prefetchL2(g + static_cast<size_t>(pf) * C, min(C, len - static_cast<uint32_t>(pf) * C));
  };
  if (producer) {
    for (; next < total && next < kRingChunks; ++next) issue(next);
    pf = next;
    prefetchTo(next + prefetchChunks);
  }

  // Prologue into the tile's slice of x (overlaps the first copies).
  {
    W beta = W(0), omega = W(0), alpha = W(0);
    bool first = true;
    if (pro.st) {
      beta = cvt<W>(pro.st->beta);
      omega = cvt<W>(pro.st->omega);
      alpha = cvt<W>(pro.st->alpha);
      first = pro.st->iter == 0;
    }
    for (int i = threadIdx.x; i < nRows; i += blockDim.x) xs[i] = pro(base + i, beta, omega, alpha, first);
  }

  int waited = 0;  // chunks known to have landed (warp 0)
  bool timedOut = false;
  auto waitTo = [&](uint32_t endByte) {
    const int need = static_cast<int>((endByte + C - 1) / C);
    for (; waited < need && !timedOut; ++waited) {
      const uint32_t bar = smemAddr(bars + (waited % kRingChunks));
      const uint32_t parity = (waited / kRingChunks) & 1;
      long long it = 0;
      while (!mbarTryWait(bar, parity))
        if (++it > kWaitLimit) {
          timedOut = true;
          break;
        }
    }
  };
  auto rdInt = [&](uint32_t o) { return *reinterpret_cast<const int*>(ring + (o & mask)); };
  auto rdVal = [&](uint32_t o) { return *reinterpret_cast<const MV*>(ring + (o & mask)); };
  auto levelEnd = [&](uint32_t o) {
    const int4 h = *reinterpret_cast<const int4*>(ring + (o & mask));
    const uint32_t k = static_cast<uint32_t>(h.x), E = static_cast<uint32_t>(h.y);
    const uint32_t rowsOff = o + 16;
    const uint32_t invOff = rowsOff + pad16u(4u * k);
    const uint32_t colsOff = invOff + (h.z ? pad16u(static_cast<uint32_t>(sizeof(MV)) * k) : 0u);
    const uint32_t valsOff = colsOff + pad16u(4u * E * k);
    return valsOff + pad16u(static_cast<uint32_t>(sizeof(MV)) * E * k);
  };

  if (waiter) {
    waitTo(16);
    if (!timedOut) {
      const int4 th = *reinterpret_cast<const int4*>(ring);
      if (th.x + th.y > 0) {
        waitTo(32);
        if (!timedOut) waitTo(levelEnd(16));
      }
    }
    if (timedOut) abortFlag = 1;
  }
  __syncthreads();
  int nL = 0, nU = 0;
  if (!abortFlag) {
    const int4 th = *reinterpret_cast<const int4*>(ring);
    nL = th.x;
    nU = th.y;
  }
  uint32_t off = 16;
  for (int lv = 0; lv < nL + nU; ++lv) {
    const int4 h = *reinterpret_cast<const int4*>(ring + (off & mask));
    const int k = h.x, E = h.y;
    const uint32_t rowsOff = off + 16;
    const uint32_t invOff = rowsOff + pad16u(4u * k);
    const uint32_t colsOff = invOff + (h.z ? pad16u(static_cast<uint32_t>(sizeof(MV)) * k) : 0u);
    const uint32_t valsOff = colsOff + pad16u(4u * E * k);
    const uint32_t end = valsOff + pad16u(static_cast<uint32_t>(sizeof(MV)) * E * k);
    const uint32_t colStride = 4u * k, valStride = static_cast<uint32_t>(sizeof(MV)) * k;
    if (!computer) {
      // The producer warp: refill consumed ring slots, then wait until the
      // next level has landed.
      if (producer) {
        const int limit = static_cast<int>(off / C) + kRingChunks;
        if (next < total && next < limit) fenceProxyAsync();
        for (; next < total && next < limit; ++next) issue(next);
        prefetchTo(next + prefetchChunks);
      }
      if (lv + 1 < nL + nU) {
        waitTo(end + 16);
        if (!timedOut) waitTo(levelEnd(end));
        if (timedOut) abortFlag = 1;
      }
    } else if (lv < nL) {
      // Forward substitution (ilu/Solver.cpp:380-411).
      for (int q = threadIdx.x; q < k; q += kComputeThreads) {
        const int il = rdInt(rowsOff + 4u * q);
        const W temp = rowDot<MV, UNROLL>(xs[il], E, colsOff + 4u * q, valsOff + static_cast<uint32_t>(sizeof(MV)) * q,
                                  colStride, valStride, xs, rdInt, rdVal);
        xs[il] = dilu ? mul(temp, cvt<W>(rdVal(invOff + static_cast<uint32_t>(sizeof(MV)) * q))) : temp;
      }
    } else {
      // Backward substitution (ilu/Solver.cpp:413-442).
      for (int q = threadIdx.x; q < k; q += kComputeThreads) {
        const int il = rdInt(rowsOff + 4u * q);
        const W temp = rowDot<MV, UNROLL>(W(0), E, colsOff + 4u * q, valsOff + static_cast<uint32_t>(sizeof(MV)) * q,
                                  colStride, valStride, xs, rdInt, rdVal);
        const W iv = cvt<W>(rdVal(invOff + static_cast<uint32_t>(sizeof(MV)) * q));
        xs[il] = dilu ? add(xs[il], mul(temp, iv)) : mul(add(xs[il], temp), iv);
      }
    }
    __syncthreads();
    if (abortFlag) break;
    off = end;
  }
  if (abortFlag) {
    if (producer) {
      atomicExch(errFlag, GR_ETIMEOUT);
      // Let the copies already issued land before the block's shared
      // memory is released (bounded).
      for (int c = waited; c < next; ++c) {
        long long it = 0;
        while (!mbarTryWait(smemAddr(bars + (c % kRingChunks)), (c / kRingChunks) & 1) && ++it < kWaitLimit) {
        }
      }
    }
    return;
  }
  for (int i = threadIdx.x; i < nRows; i += blockDim.x) y[base + i] = xs[i];
}

template <class MV>
__global__ void streamPackKernel(MV* __restrict__ stream, const int* __restrict__ valPos,
                                 const int* __restrict__ valSrc, long long nVal, const MV* __restrict__ F,
                                 const int* __restrict__ invPos, const int* __restrict__ invSrc, long long nInv,
                                 const MV* __restrict__ inv) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < nVal; i += stride) {
    const int s = valSrc[i];
    stream[valPos[i]] = s >= 0 ? F[s] : MV(0);
  }
  for (long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; j < nInv; j += stride)
    stream[invPos[j]] = inv[invSrc[j]];
}

}  // namespace dev

// ---------------------------------------------------------------------------
static_assert(dev::kRingChunks == kRingChunksHost, "ring geometry shared with the host checker");

int iluStreamRingLog2(const SweepStream& S, int requested) {
  const int need = ringLog2ForLevel(S.maxSpanBytes);
  return requested > need ? requested : need;
}

size_t iluStreamSmem(const DeviceMatrix& A, const SweepStream& S, DType W, int ringLog2) {
  const int lg = iluStreamRingLog2(S, ringLog2);
  if (lg > 17) return 0;    // rings above 128 KB: use the level-schedule kernel
  return 128 + (size_t(1) << lg) + static_cast<size_t>(A.host->maxTileRows) * dtypeSize(W);
}

void launchPackBytes(DeviceMatrix& A, const void* templ, i64 bytes, const int* valPos, const int* valSrc, i64 nVal,
                     const int* invPos, const int* invSrc, i64 nInv, void* stream, const void* F, const void* inv,
                     cudaStream_t s) {
  GR_CUDA(cudaMemcpyAsync(stream, templ, bytes, cudaMemcpyDeviceToDevice, s));
  const int blocks = static_cast<int>(std::max<i64>(1, std::min<i64>(A.redBlocks, (std::max(nVal, nInv) + 255) / 256)));
  if (A.vt == DType::F32)
    dev::streamPackKernel<float><<<blocks, 256, 0, s>>>(static_cast<float*>(stream), valPos, valSrc, nVal,
                                                        static_cast<const float*>(F), invPos, invSrc, nInv,
                                                        static_cast<const float*>(inv));
  else
    dev::streamPackKernel<double><<<blocks, 256, 0, s>>>(static_cast<double*>(stream), valPos, valSrc, nVal,
                                                         static_cast<const double*>(F), invPos, invSrc, nInv,
                                                         static_cast<const double*>(inv));
  checkLaunch("stream_pack");
}

void launchStreamPack(DeviceMatrix& A, const SweepStream& S, void* stream, const void* F, const void* inv,
                      cudaStream_t s) {
  launchPackBytes(A, S.templ.get(), S.bytes, S.valPos.as<int>(), S.valSrc.as<int>(), S.nVal, S.invPos.as<int>(),
                  S.invSrc.as<int>(), S.nInv, stream, F, inv, s);
}

namespace {
template <class MV, class W>
void streamApplyT(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu, const PrologueArgs& p,
                  void* y, const StreamTuning& tune, cudaStream_t s) {
  const int lg = iluStreamRingLog2(S, tune.ringLog2);
  const size_t smem = iluStreamSmem(A, S, dtypeOf<W>(), tune.ringLog2);
  auto kernel = tune.unroll ? dev::iluStreamKernel<MV, W, true> : dev::iluStreamKernel<MV, W, false>;
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
  const int pf = tune.prefetchChunks < 0 ? dev::kPrefetchChunks : tune.prefetchChunks;
  dev::SPro<W> pro{static_cast<int>(p.kind), static_cast<const W*>(p.b), static_cast<const W*>(p.r),
                   static_cast<W*>(p.pOrS), static_cast<const W*>(p.v), p.st};
  kernel<<<A.P, dev::kStreamThreads, smem, s>>>(static_cast<const unsigned char*>(stream), S.tileOffset.as<long long>(),
                                A.tileStart.as<int>(), lg, pf, dilu, pro, static_cast<W*>(y), A.errFlag.as<int>());
  checkLaunch("ilu_stream");
}
}  // namespace

void launchIluStream(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu,
                     const PrologueArgs& pro, void* y, DType W, const StreamTuning& tune, cudaStream_t s) {
  if (A.vt == DType::F32 && W == DType::F32) streamApplyT<float, float>(A, S, stream, dilu, pro, y, tune, s);
  else if (A.vt == DType::F32 && W == DType::F64)
    streamApplyT<float, double>(A, S, stream, dilu, pro, y, tune, s);
  else if (A.vt == DType::F64 && W == DType::F64)
    streamApplyT<double, double>(A, S, stream, dilu, pro, y, tune, s);
  else fail(GR_EUNSUPPORTED, "ILU with float64 coefficients needs float64 vectors");
}

}  // namespace gr

// Block-ILU(0) / DILU substitution through a host-scheduled shared-memory
// ring (ilu/Solver.cpp:367-550, level by level; same arithmetic and order as
// the other substitution kernels).
//
// One thread block per group of consecutive tiles, run in lockstep (level l
// of the block is level l of each of its tiles). The level blocks (LevelRing, device.hpp)
// are copied from global memory into a shared-memory ring with one bulk
// asynchronous copy per level (cp.async.bulk, completion on one of
// kRingBarriers mbarriers; a single-CTA bulk copy: a block copies only its
// own tile's bytes from this GPU's memory). The host fixed each level's ring offset and
// the level after which its copy is issued, so the kernel does no ring
// arithmetic: a level's rows, inverse diagonal and (column, value) entries
// sit at fixed offsets. Producer and consumers form a pipeline over
// kRingBarriers pairs of mbarriers: the producer warp issues level j's copy
// (completing on full[j % 16]) once level issueAfter(j) has been released
// (empty[...]). The compute warps compute level l's rows from shared memory
// while a waiting warp waits for full[(l + 1) % 16]; they meet at a barrier
// of their own that ends level l, after which the waiting warp releases
// level l. Neither the producer's copies nor the mbarrier waits
// and arrivals sit on the compute warps' per-level chain.
//
// Every wait is bounded; when one runs out the block records GR_ETIMEOUT in
// the matrix's error word, the other waits give up, and the issuing lane
// waits (bounded) for the copies still in flight before the block exits.
#include <algorithm>
#include <climits>

#include "bulk.cuh"
#include "device.hpp"
#include "devmath.cuh"
#include "krylov.hpp"
#include "sell.cuh"

namespace gr {
namespace dev {

// Compute warps, a waiting warp and a producer warp per block. Fewer
// compute warps mean fewer instructions and barrier arrivals per level; with
// float vectors (seven blocks an SM at 192^3, 2048 tiles) two were fastest on
// B200 (116.8 us against 123.0 for one, 117.0 for three, 121 for four, 125.5
// for six); double vectors take twice the shared memory, so fewer blocks
// share an SM, and four were faster for them.
template <class W>
struct RingShape {
  static constexpr int compute = sizeof(W) == 4 ? 64 : 128;
  static constexpr int levelSync = compute + 32;  // compute warps + waiting warp
  static constexpr int threads = levelSync + 32;
};
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

// A level of the ring as the compute warps see it.
template <class MV, bool COMPACT>
struct RingLevel {
  int k, E;
  bool upper, rec;
  const unsigned char* blk;  // the level block in the ring
  uint32_t inv, ents, vals;  // offsets of its inverse diagonal, entries (columns) and values
  __device__ __forceinline__ int row(int q) const {
    return COMPACT ? static_cast<int>(reinterpret_cast<const uint16_t*>(blk)[q]) : reinterpret_cast<const int*>(blk)[q];
  }
  __device__ __forceinline__ MV invDiag(int q) const { return reinterpret_cast<const MV*>(blk + inv)[q]; }
  // Entry e of row q.
  __device__ __forceinline__ void entry(int e, int q, int& c, MV& v) const {
    const int idx = e * k + q;
    if (COMPACT) {
      c = reinterpret_cast<const uint16_t*>(blk + ents)[idx];
      v = reinterpret_cast<const MV*>(blk + vals)[idx];
    } else {
      loadEntry<MV>(blk + ents + (sizeof(MV) == 4 ? 8 : 16) * idx, c, v);
    }
  }
};
// The level's view from its table entry (RingLevelCode): the inverse
// diagonal follows the row ids, the values (compact layout) the columns.
template <class MV, bool COMPACT>
__device__ __forceinline__ RingLevel<MV, COMPACT> ringLevelAt(const int4 m, const unsigned char* ring) {
  RingLevel<MV, COMPACT> lv;
  lv.k = RingLevelCode::k(m);
  lv.E = RingLevelCode::E(m);
  lv.upper = RingLevelCode::upper(m);
  lv.rec = COMPACT && sizeof(MV) == 4 && RingLevelCode::record(m);
  lv.blk = ring + RingLevelCode::ringOffset(m);
  lv.inv = ((COMPACT ? 2u : 4u) * static_cast<uint32_t>(lv.k) + 15u) & ~15u;
  lv.ents = RingLevelCode::ents(m);
  lv.vals = COMPACT ? lv.ents + ((2u * static_cast<uint32_t>(lv.E) * static_cast<uint32_t>(lv.k) + 15u) & ~15u)
                    : lv.ents;
  return lv;
}

// Row q of a record level (float values, 3 entries): one 16-byte load
// {v0, v1, v2, c0 | c1 << 16} and one 4- or 8-byte load {c2 | row << 16,
// inverse diagonal}.
struct RowRecord {
  int row, c[3];
  float v[3], inv;
};
template <class MV, bool COMPACT>
__device__ __forceinline__ RowRecord ringRecord(const RingLevel<MV, COMPACT>& lv, int q, bool hasInv) {
  RowRecord r;
  const float4 a = reinterpret_cast<const float4*>(lv.blk)[q];
  // The {c2 | row, inverse diagonal} words follow the k records (the host
  // lays record levels out so that ents == 16 k; the ring check verifies
  // it), so their address comes from k without decoding the table entry.
  const unsigned char* words = lv.blk + 16 * lv.k;
  uint32_t w2;
  if (hasInv) {
    const uint2 b = reinterpret_cast<const uint2*>(words)[q];
    w2 = b.x;
    r.inv = __uint_as_float(b.y);
  } else {
    w2 = reinterpret_cast<const uint32_t*>(words)[q];
    r.inv = 0.0f;
  }
  const uint32_t w01 = __float_as_uint(a.w);
  r.c[0] = static_cast<int>(w01 & 0xFFFFu);
  r.c[1] = static_cast<int>(w01 >> 16);
  r.c[2] = static_cast<int>(w2 & 0xFFFFu);
  r.row = static_cast<int>(w2 >> 16);
  r.v[0] = a.x;
  r.v[1] = a.y;
  r.v[2] = a.z;
  return r;
}
// temp -= v0 x[c0], v1 x[c1], v2 x[c2], in order (x loads first).
template <class W>
__device__ __forceinline__ W recordDot(W temp, const RowRecord& r, const W* xs) {
  const W x0 = xs[r.c[0]], x1 = xs[r.c[1]], x2 = xs[r.c[2]];
  temp = sub(temp, mul(cvt<W>(r.v[0]), x0));
  temp = sub(temp, mul(cvt<W>(r.v[1]), x1));
  return sub(temp, mul(cvt<W>(r.v[2]), x2));
}

// temp -= sum_e value_e * xs[column_e] over row q's E entries in order.
// Padding entries (column = the zero slot, value 0) leave temp unchanged.
// Rows of up to four entries load all their entries, then all x values,
// before the arithmetic.
template <bool UNROLL, class MV, bool COMPACT, class W>
__device__ __forceinline__ W ringRowDot(W temp, const RingLevel<MV, COMPACT>& lv, int q, int zeroSlot,
                                        const W* xs) {
  if (UNROLL && lv.E <= 4) {
    int c[4];
    MV v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (e < lv.E) {
        lv.entry(e, q, c[e], v[e]);
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
      if (e < lv.E) temp = sub(temp, mul(cvt<W>(v[e]), xv[e]));
    return temp;
  }
  for (int e = 0; e < lv.E; ++e) {
    int c;
    MV v;
    lv.entry(e, q, c, v);
    temp = sub(temp, mul(cvt<W>(v), xs[c]));
  }
  return temp;
}

// CW compute warps (0: RingShape's default for W); the waiting warp
// (WAITER) and the producer warp follow them. Without the waiting warp the
// compute warps wait for each next level themselves and release the level
// they finished.
template <int CW, class W>
constexpr int ringComputeThreads() {
  return CW > 0 ? 32 * CW : RingShape<W>::compute;
}
// PRODUCER false (with WAITER): no producer warp; the waiting warp's first
// lane issues the copies whose ring space level l freed right after the
// barrier that ends level l (the host schedule issues every level's copy at
// least one level before it is needed, so the copy the waiting warp waits
// for has always been issued), and no empty barriers are used.
//
// With the waiting warp a level ends with a plain named barrier: the waiting
// warp, the only one that can decide to stop, writes the level after which
// every thread stops (once, before that level's barrier), and every thread
// reads it after the barrier. On B200 this ran 2-9 % faster than a barrier
// with an OR reduction carrying the decision (bar.red.or: 167 cycles against
// 120 for bar.sync among three warps, measured alone).
template <class MV, class W, bool UNROLL, bool COMPACT, int CW = 0, bool WAITER = true, bool PRODUCER = true>
__global__ void __launch_bounds__(ringComputeThreads<CW, W>() + (WAITER ? 32 : 0) + (PRODUCER ? 32 : 0)) iluRingKernel(
    const unsigned char* __restrict__ stream,
                                                               const long long* __restrict__ tileOffset,
                                                               const int4* __restrict__ meta,
                                                               const int* __restrict__ tileLevel,
                                                               const int* __restrict__ blockStart, int ringBytes,
                                                               int metaLevels, uint32_t l2Ahead, bool dilu,
                                                               SPro<W> pro, W* __restrict__ y, int* errFlag,
                                                               bool pairRows) {
  constexpr int kRingCompute = ringComputeThreads<CW, W>();
  constexpr int kRingLevelSync = kRingCompute + (WAITER ? 32 : 0);
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int abortFlag, consumedLevels;
  // The level after whose barrier every thread stops (waiting warp only).
  __shared__ int stopAt;
  const volatile int* stopAtV = &stopAt;
  const KState* st = pro.state();
  if (st && st->done) return;
  const int T = blockIdx.x;
  const int base = blockStart[T];
  const int nRows = blockStart[T + 1] - base;
  const int lv0 = tileLevel[T];
  const int L = tileLevel[T + 1] - lv0;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);  // level landed, one per barrier slot
  uint64_t* empty = full + kRingBarriers;              // level consumed by the compute warps
  uint64_t* tableBar = empty + kRingBarriers;
  int4* mt = reinterpret_cast<int4*>(smem + kRingHeader);
  unsigned char* ring = smem + kRingHeader + 16 * metaLevels;
  W* xs = reinterpret_cast<W*>(ring + ringBytes);
  const unsigned char* g = stream + tileOffset[T];
  static_assert(WAITER || PRODUCER, "a ring kernel without a waiting warp needs the producer warp");
  // The issuing lane: the producer warp's first lane, or the waiting warp's.
  const bool lead = threadIdx.x == (PRODUCER ? kRingLevelSync : kRingCompute);
  const volatile int* abortV = &abortFlag;

  if (lead) {
    abortFlag = 0;
    stopAt = INT_MAX;
    consumedLevels = L;
    for (int i = 0; i < kRingBarriers; ++i) {
      mbarInit(smemAddr(full + i), 1);
      mbarInit(smemAddr(empty + i), 1);
    }
    mbarInit(smemAddr(tableBar), 1);
    fenceBarrierInit();
    const uint32_t tb = static_cast<uint32_t>(L) * 16u;
    mbarExpectTx(smemAddr(tableBar), tb);
    bulkLoad(smemAddr(mt), meta + static_cast<size_t>(lv0), tb, smemAddr(tableBar));
  }
  // Prologue into the block's slice of x while the level table lands; the
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
    // kPro rows a thread at once, all loads before any store. (Eight rows
    // a thread ran no faster on B200 and took the kernel from 32 to 48
    // registers, which caps the tiles resident per SM at 10.)
    constexpr int kPro = 4;
    const int bd = static_cast<int>(blockDim.x);
    for (int i0 = threadIdx.x; i0 < nRows; i0 += kPro * bd) {
      W v[kPro];
      pro.template rows<kPro>(base + i0, bd, base + nRows, beta, omega, alpha, first, v);
#pragma unroll
      for (int j = 0; j < kPro; ++j)
        if (i0 + j * bd < nRows) xs[i0 + j * bd] = v[j];
    }
    if (lead) xs[nRows] = W(0);
  }
  __syncthreads();  // barriers initialised, x slice written

  int issued = 0;  // issuing lane: levels whose copies were issued
  uint32_t src = 0;
  // Issuing lane without a producer warp: the copies of every level j with
  // issueAfter(j) <= done, in order (issueAfter never decreases along the
  // levels; the next one is kept in a register).
  int nextAfter = INT_MAX;
  auto issueUpTo = [&](int done) {
    while (nextAfter <= done) {
      const int4 m = mt[issued];
      const uint32_t bytes = RingLevelCode::bytes(m);
      const uint32_t bar = smemAddr(full + issued % kRingBarriers);
      mbarExpectTx(bar, bytes);
      bulkLoad(smemAddr(ring + RingLevelCode::ringOffset(m)), g + src, bytes, bar);
      src += bytes;
      ++issued;
      nextAfter = issued < L ? RingLevelCode::issueAfter(mt[issued]) : INT_MAX;
    }
  };
  if (PRODUCER && threadIdx.x >= kRingLevelSync) {
    // Producer: copies the levels in order, level j once level
    // issueAfter(j) has been released on its empty barrier (after the
    // barrier that ended it, so every read of it is done). It runs ahead of
    // the compute warps by as much as the ring allows and takes no part in
    // their per-level barrier.
    if (lead) {
      if (!mbarWaitBounded(smemAddr(tableBar), 0, abortV)) {
        abortFlag = 1;
      } else {
        uint32_t pf = 0;
        const uint32_t tileBytes = static_cast<uint32_t>(tileOffset[T + 1] - tileOffset[T]);
        for (; issued < L && !*abortV; ++issued) {
          const int4 m = mt[issued];
          const int ia = RingLevelCode::issueAfter(m);
          if (ia >= 0 && !mbarWaitBounded(smemAddr(empty + ia % kRingBarriers), (ia / kRingBarriers) & 1, abortV)) {
            abortFlag = 1;
            break;
          }
          const uint32_t bytes = RingLevelCode::bytes(m);
          const uint32_t bar = smemAddr(full + issued % kRingBarriers);
          mbarExpectTx(bar, bytes);
          bulkLoad(smemAddr(ring + RingLevelCode::ringOffset(m)), g + src, bytes, bar);
          src += bytes;
          if (pf < src) pf = src;
          const uint32_t until = min(tileBytes, src + l2Ahead);
          if (pf < until) {
            prefetchL2(g + pf, until - pf);
            pf = until;
          }
        }
      }
    }
  } else if (WAITER && threadIdx.x >= kRingCompute) {
    // Waiting warp: before the barrier that ends level l it waits until
    // level l + 1 has landed (so the barrier also publishes the copy to the
    // compute warps); after it, it releases level l (or, without a producer
    // warp, issues the copies that level l's release allows).
    bool ok = mbarWaitBounded(smemAddr(tableBar), 0, abortV);
    if (!PRODUCER && ok && lead) {
      nextAfter = L > 0 ? RingLevelCode::issueAfter(mt[0]) : INT_MAX;
      issueUpTo(-1);
    }
    ok = ok && (L == 0 || mbarWaitBounded(smemAddr(full), 0, abortV));
    if (!ok) abortFlag = 1;
    bool stop;
    if (!ok) stopAt = -1;
    namedBarSync(1, kRingLevelSync);
    stop = *stopAtV <= -1;
    if (stop && threadIdx.x == kRingCompute) consumedLevels = 0;
    for (int l = 0; !stop && l < L; ++l) {
      bool bad = false;
      if (l + 1 < L && !mbarWaitBounded(smemAddr(full + (l + 1) % kRingBarriers), ((l + 1) / kRingBarriers) & 1, abortV)) {
        abortFlag = 1;
        bad = true;
      }
      if (bad || *abortV != 0) stopAt = l;
      namedBarSync(1, kRingLevelSync);
      stop = *stopAtV <= l;
      if (threadIdx.x == kRingCompute) {
        if constexpr (PRODUCER) mbarArrive(smemAddr(empty + l % kRingBarriers));
        else if (!stop) issueUpTo(l);
        if (stop) consumedLevels = l + 1;
      }
    }
  } else {
    // Compute warps: level l, whose block the waiting warp (or, without
    // one, each compute thread) saw land before the previous barrier.
    bool stop;
    if constexpr (WAITER) {
      namedBarSync(1, kRingLevelSync);
      stop = *stopAtV <= -1;
    } else {
      const bool ok = mbarWaitBounded(smemAddr(tableBar), 0, abortV) &&
                      (L == 0 || mbarWaitBounded(smemAddr(full), 0, abortV));
      if (!ok) abortFlag = 1;
      stop = namedBarOr(1, kRingCompute, !ok);
      if (stop && threadIdx.x == 0) consumedLevels = 0;
    }
    for (int l = 0; !stop && l < L; ++l) {
      const int4 m = mt[l];
      const RingLevel<MV, COMPACT> cur = ringLevelAt<MV, COMPACT>(m, ring);
      if (cur.rec) {
        // Record level (7-point lower or upper part): the same operations
        // as below, from two loads a row.
        const bool hasInv = cur.upper || dilu;
        int q0 = threadIdx.x;
        if (pairRows) {
          // Two rows of the level a thread at once (rows of one level never
          // read each other): both rows' loads before either store.
          for (; q0 + kRingCompute < cur.k; q0 += 2 * kRingCompute) {
            const RowRecord ra = ringRecord(cur, q0, hasInv);
            const RowRecord rb = ringRecord(cur, q0 + kRingCompute, hasInv);
            if (!cur.upper) {
              const W ta = recordDot(xs[ra.row], ra, xs);
              const W tb = recordDot(xs[rb.row], rb, xs);
              xs[ra.row] = dilu ? mul(ta, cvt<W>(ra.inv)) : ta;
              xs[rb.row] = dilu ? mul(tb, cvt<W>(rb.inv)) : tb;
            } else {
              const W ta = recordDot(W(0), ra, xs), tb = recordDot(W(0), rb, xs);
              const W xa = xs[ra.row], xb = xs[rb.row];
              const W ia = cvt<W>(ra.inv), ib = cvt<W>(rb.inv);
              xs[ra.row] = dilu ? add(xa, mul(ta, ia)) : mul(add(xa, ta), ia);
              xs[rb.row] = dilu ? add(xb, mul(tb, ib)) : mul(add(xb, tb), ib);
            }
          }
        }
        for (int q = q0; q < cur.k; q += kRingCompute) {
          const RowRecord r = ringRecord(cur, q, hasInv);
          if (!cur.upper) {
            const W temp = recordDot(xs[r.row], r, xs);
            xs[r.row] = dilu ? mul(temp, cvt<W>(r.inv)) : temp;
          } else {
            const W temp = recordDot(W(0), r, xs);
            const W iv = cvt<W>(r.inv);
            xs[r.row] = dilu ? add(xs[r.row], mul(temp, iv)) : mul(add(xs[r.row], temp), iv);
          }
        }
      } else if (!cur.upper) {
        // Forward substitution (ilu/Solver.cpp:380-411).
        for (int q = threadIdx.x; q < cur.k; q += kRingCompute) {
          const int il = cur.row(q);
          const W temp = ringRowDot<UNROLL>(xs[il], cur, q, nRows, xs);
          xs[il] = dilu ? mul(temp, cvt<W>(cur.invDiag(q))) : temp;
        }
      } else {
        // Backward substitution (ilu/Solver.cpp:413-442).
        for (int q = threadIdx.x; q < cur.k; q += kRingCompute) {
          const int il = cur.row(q);
          const W temp = ringRowDot<UNROLL>(W(0), cur, q, nRows, xs);
          const W iv = cvt<W>(cur.invDiag(q));
          xs[il] = dilu ? add(xs[il], mul(temp, iv)) : mul(add(xs[il], temp), iv);
        }
      }
      if constexpr (WAITER) {
        namedBarSync(1, kRingLevelSync);
        stop = *stopAtV <= l;
      } else {
        bool bad = false;
        if (l + 1 < L &&
            !mbarWaitBounded(smemAddr(full + (l + 1) % kRingBarriers), ((l + 1) / kRingBarriers) & 1, abortV)) {
          abortFlag = 1;
          bad = true;
        }
        stop = namedBarOr(1, kRingCompute, bad || *abortV != 0);
        if (threadIdx.x == 0) {
          mbarArrive(smemAddr(empty + l % kRingBarriers));
          if (stop) consumedLevels = l + 1;
        }
      }
    }
  }
  __syncthreads();
  if (abortFlag) {
    if (lead) {
      atomicExch(errFlag, GR_ETIMEOUT);
      // Let the copies already issued land before the block's shared memory
      // is released (bounded). Each barrier has at most one such copy: level
      // j + kRingBarriers is issued only after level j was consumed.
      mbarWaitBounded(smemAddr(tableBar), 0);
      for (int j = consumedLevels; j < issued; ++j)
        mbarWaitBounded(smemAddr(full + j % kRingBarriers), (j / kRingBarriers) & 1);
    }
    return;
  }
  for (int i = threadIdx.x; i < nRows; i += blockDim.x) y[base + i] = xs[i];
}

// One Gauss-Seidel sweep of every tile (gauss-seidel/Solver.cpp:45-86)
// through a Gauss-Seidel level ring: rows in ascending tile-local order, as
// the lower levels, each x_i = (seed_i - sum_j a_ij x_j) / d_i over the row's
// entries in tile-local order, where x_j is this sweep's value for earlier
// rows of the tile and the sweep-start value for later rows and for halo
// cells. The same producer / waiting / compute warp pipeline as
// iluRingKernel copies the level blocks (rows, diagonal, slots, values); the
// tile's x lives in shared memory as [this sweep | sweep start | halo |
// zero], so every entry is one shared-memory read at a slot the host fixed.
// The prologue fills the sweep-start values and halo cells from xin (zeros
// when xinZero) and, with seedB, the right-hand side from the fused
// PBiCGStab prologue (which also writes p or s).
// Vectors are stored in X; rows are computed in W, each new value rounded to
// X as it is stored (the working type of gauss-seidel/Solver.cpp:65-84).
template <class X, class W>
__device__ __forceinline__ W storeRound(W v) {
  return cvt<W>(cvt<X>(v));
}
template <class MV, class X, class W, bool COMPACT>
__global__ void __launch_bounds__(RingShape<W>::threads) gsRingKernel(
    const unsigned char* __restrict__ stream, const long long* __restrict__ tileOffset, const int4* __restrict__ meta,
    const int* __restrict__ tileLevel, const int* __restrict__ tileStart, const int* __restrict__ haloStart,
    const int* __restrict__ haloSrc, int ringBytes, int metaLevels, bool seedB, SPro<X> pro,
    const X* __restrict__ xin, bool xinZero, X* __restrict__ xout, int* errFlag, bool inPlace, bool dropHalo) {
  constexpr int kRingCompute = RingShape<W>::compute;
  constexpr int kRingLevelSync = RingShape<W>::levelSync;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int abortFlag, consumedLevels;
  __shared__ int stopAt;  // the level after whose barrier every thread stops (waiting warp only)
  const volatile int* stopAtV = &stopAt;
  const KState* st = pro.state();
  if (st && st->done) return;
  const int T = blockIdx.x;
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  const int h0 = haloStart[T];
  const int nHalo = haloStart[T + 1] - h0;
  const int lv0 = tileLevel[T];
  const int L = tileLevel[T + 1] - lv0;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kRingBarriers;
  uint64_t* tableBar = empty + kRingBarriers;
  int4* mt = reinterpret_cast<int4*>(smem + kRingHeader);
  unsigned char* ring = smem + kRingHeader + 16 * metaLevels;
  W* xs = reinterpret_cast<W*>(ring + ringBytes);  // this sweep | sweep start | halo | zero
  const int s0 = inPlace ? 0 : nRows;               // start values (in place: this sweep's slots)
  const int hb = s0 + nRows;                        // halo
  W* rhs = xs + hb + nHalo + 1;
  const unsigned char* g = stream + tileOffset[T];
  const bool lead = threadIdx.x == kRingLevelSync;
  const volatile int* abortV = &abortFlag;

  if (lead) {
    abortFlag = 0;
    stopAt = INT_MAX;
    consumedLevels = L;
    for (int i = 0; i < kRingBarriers; ++i) {
      mbarInit(smemAddr(full + i), 1);
      mbarInit(smemAddr(empty + i), 1);
    }
    mbarInit(smemAddr(tableBar), 1);
    fenceBarrierInit();
    const uint32_t tb = static_cast<uint32_t>(L) * 16u;
    mbarExpectTx(smemAddr(tableBar), tb);
    bulkLoad(smemAddr(mt), meta + static_cast<size_t>(lv0), tb, smemAddr(tableBar));
  }
  {
    const int bd = static_cast<int>(blockDim.x);
    if (seedB || pro.kind != static_cast<int>(Prologue::Plain)) {
      X beta = X(0), omega = X(0), alpha = X(0);
      bool first = true;
      if (st) {
        beta = cvt<X>(st->beta);
        omega = cvt<X>(st->omega);
        alpha = cvt<X>(st->alpha);
        first = st->iter == 0;
      }
      constexpr int kPro = 4;  // rows a thread at once, loads before stores
      for (int i0 = threadIdx.x; i0 < nRows; i0 += kPro * bd) {
        X v[kPro];
        pro.template rows<kPro>(base + i0, bd, base + nRows, beta, omega, alpha, first, v);
        if (seedB) {
#pragma unroll
          for (int j = 0; j < kPro; ++j)
            if (i0 + j * bd < nRows) rhs[i0 + j * bd] = cvt<W>(v[j]);
        }
      }
    }
    for (int i = threadIdx.x; i < nRows; i += bd) xs[s0 + i] = xinZero ? W(0) : cvt<W>(xin[base + i]);
    if (xinZero || dropHalo) {
      for (int h = threadIdx.x; h < nHalo; h += bd) xs[hb + h] = W(0);
    } else {
      // Four halo cells a thread: their source indices, then their values.
      constexpr int kH = 4;
      for (int h = threadIdx.x; h < nHalo; h += kH * bd) {
        int src[kH];
#pragma unroll
        for (int j = 0; j < kH; ++j) src[j] = h + j * bd < nHalo ? haloSrc[h0 + h + j * bd] : -1;
        W hv[kH];
#pragma unroll
        for (int j = 0; j < kH; ++j) hv[j] = src[j] >= 0 ? cvt<W>(xin[src[j]]) : W(0);
#pragma unroll
        for (int j = 0; j < kH; ++j)
          if (src[j] >= 0) xs[hb + h + j * bd] = hv[j];
      }
    }
    if (lead) xs[hb + nHalo] = W(0);
  }
  __syncthreads();

  int issued = 0;
  if (threadIdx.x >= kRingLevelSync) {
    if (lead) {
      if (!mbarWaitBounded(smemAddr(tableBar), 0, abortV)) {
        abortFlag = 1;
      } else {
        uint32_t src = 0;
        for (; issued < L && !*abortV; ++issued) {
          const int4 m = mt[issued];
          const int ia = RingLevelCode::issueAfter(m);
          if (ia >= 0 && !mbarWaitBounded(smemAddr(empty + ia % kRingBarriers), (ia / kRingBarriers) & 1, abortV)) {
            abortFlag = 1;
            break;
          }
          const uint32_t bytes = RingLevelCode::bytes(m);
          const uint32_t bar = smemAddr(full + issued % kRingBarriers);
          mbarExpectTx(bar, bytes);
          bulkLoad(smemAddr(ring + RingLevelCode::ringOffset(m)), g + src, bytes, bar);
          src += bytes;
        }
      }
    }
  } else if (threadIdx.x >= kRingCompute) {
    bool ok = mbarWaitBounded(smemAddr(tableBar), 0, abortV) && (L == 0 || mbarWaitBounded(smemAddr(full), 0, abortV));
    if (!ok) {
      abortFlag = 1;
      stopAt = -1;
    }
    namedBarSync(1, kRingLevelSync);
    bool stop = *stopAtV <= -1;
    if (stop && threadIdx.x == kRingCompute) consumedLevels = 0;
    for (int l = 0; !stop && l < L; ++l) {
      bool bad = false;
      if (l + 1 < L &&
          !mbarWaitBounded(smemAddr(full + (l + 1) % kRingBarriers), ((l + 1) / kRingBarriers) & 1, abortV)) {
        abortFlag = 1;
        bad = true;
      }
      if (bad || *abortV != 0) stopAt = l;
      namedBarSync(1, kRingLevelSync);
      stop = *stopAtV <= l;
      if (threadIdx.x == kRingCompute) {
        mbarArrive(smemAddr(empty + l % kRingBarriers));
        if (stop) consumedLevels = l + 1;
      }
    }
  } else {
    namedBarSync(1, kRingLevelSync);
    bool stop = *stopAtV <= -1;
    for (int l = 0; !stop && l < L; ++l) {
      const RingLevel<MV, COMPACT> cur = ringLevelAt<MV, COMPACT>(mt[l], ring);
      if (cur.rec) {
        for (int q = threadIdx.x; q < cur.k; q += kRingCompute) {
          const RowRecord r = ringRecord(cur, q, true);
          const W d = cvt<W>(r.inv);
          const W sum = recordDot(seedB ? rhs[r.row] : d, r, xs);
          xs[r.row] = storeRound<X>(dvd(sum, d));
        }
        namedBarSync(1, kRingLevelSync);
        stop = *stopAtV <= l;
        continue;
      }
      for (int q = threadIdx.x; q < cur.k; q += kRingCompute) {
        const int il = cur.row(q);
        const W d = cvt<W>(cur.invDiag(q));
        W sum = seedB ? rhs[il] : d;
        if (cur.E <= 8) {
          // Every entry's slot and value first, then the x values, then the
          // sum in order: the loads overlap.
          int c[8];
          MV v[8];
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (e < cur.E) cur.entry(e, q, c[e], v[e]);
          W xv[8];
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (e < cur.E) xv[e] = xs[c[e]];
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (e < cur.E) sum = sub(sum, mul(cvt<W>(v[e]), xv[e]));
        } else {
          for (int e = 0; e < cur.E; ++e) {
            int c;
            MV v;
            cur.entry(e, q, c, v);
            sum = sub(sum, mul(cvt<W>(v), xs[c]));
          }
        }
        xs[il] = storeRound<X>(dvd(sum, d));
      }
      namedBarSync(1, kRingLevelSync);
      stop = *stopAtV <= l;
    }
  }
  __syncthreads();
  if (abortFlag) {
    if (lead) {
      atomicExch(errFlag, GR_ETIMEOUT);
      mbarWaitBounded(smemAddr(tableBar), 0);
      for (int j = consumedLevels; j < issued; ++j)
        mbarWaitBounded(smemAddr(full + j % kRingBarriers), (j / kRingBarriers) & 1);
    }
    return;
  }
  for (int i = threadIdx.x; i < nRows; i += blockDim.x) xout[base + i] = cvt<X>(xs[i]);
}

// Level l's rows for thread t of `stride` threads: the substitution of
// iluRingKernel's compute warps (same operations, same order).
template <int STRIDE, class MV, class W, bool COMPACT>
__device__ __forceinline__ void iluLevelRows(const RingLevel<MV, COMPACT>& cur, int t, int nRows, bool dilu,
                                             bool pairRows, W* xs) {
  if (cur.rec) {
    const bool hasInv = cur.upper || dilu;
    int q0 = t;
    if (pairRows) {
      for (; q0 + STRIDE < cur.k; q0 += 2 * STRIDE) {
        const RowRecord ra = ringRecord(cur, q0, hasInv);
        const RowRecord rb = ringRecord(cur, q0 + STRIDE, hasInv);
        if (!cur.upper) {
          const W ta = recordDot(xs[ra.row], ra, xs);
          const W tb = recordDot(xs[rb.row], rb, xs);
          xs[ra.row] = dilu ? mul(ta, cvt<W>(ra.inv)) : ta;
          xs[rb.row] = dilu ? mul(tb, cvt<W>(rb.inv)) : tb;
        } else {
          const W ta = recordDot(W(0), ra, xs), tb = recordDot(W(0), rb, xs);
          const W xa = xs[ra.row], xb = xs[rb.row];
          const W ia = cvt<W>(ra.inv), ib = cvt<W>(rb.inv);
          xs[ra.row] = dilu ? add(xa, mul(ta, ia)) : mul(add(xa, ta), ia);
          xs[rb.row] = dilu ? add(xb, mul(tb, ib)) : mul(add(xb, tb), ib);
        }
      }
    }
    for (int q = q0; q < cur.k; q += STRIDE) {
      const RowRecord r = ringRecord(cur, q, hasInv);
      if (!cur.upper) {
        const W temp = recordDot(xs[r.row], r, xs);
        xs[r.row] = dilu ? mul(temp, cvt<W>(r.inv)) : temp;
      } else {
        const W temp = recordDot(W(0), r, xs);
        const W iv = cvt<W>(r.inv);
        xs[r.row] = dilu ? add(xs[r.row], mul(temp, iv)) : mul(add(xs[r.row], temp), iv);
      }
    }
  } else if (!cur.upper) {
    for (int q = t; q < cur.k; q += STRIDE) {
      const int il = cur.row(q);
      const W temp = ringRowDot<true>(xs[il], cur, q, nRows, xs);
      xs[il] = dilu ? mul(temp, cvt<W>(cur.invDiag(q))) : temp;
    }
  } else {
    for (int q = t; q < cur.k; q += STRIDE) {
      const int il = cur.row(q);
      const W temp = ringRowDot<true>(W(0), cur, q, nRows, xs);
      const W iv = cvt<W>(cur.invDiag(q));
      xs[il] = dilu ? add(xs[il], mul(temp, iv)) : mul(add(xs[il], temp), iv);
    }
  }
}

// ILU(0) / DILU substitution with one warp per tile (same arithmetic and
// order as iluRingKernel). Each warp owns a slice of shared memory: its
// tile's kRingBarriers completion mbarriers, level table, level ring and x
// slice. The warp waits for level l's block on its own barrier, computes
// the level's rows, meets its lanes with __syncwarp (no block-wide barrier,
// no waiting or producer warp), and then lane 0 issues the bulk copies of
// every later level whose ring space was held by level l or earlier (the
// host schedule's issueAfter). The prologue keeps 16 (float) or 8 (double)
// rows a lane in flight. Waits are bounded as in iluRingKernel.
template <class MV, class W, bool COMPACT>
__global__ void __launch_bounds__(256) iluWarpRingKernel(const unsigned char* __restrict__ stream,
                                                          const long long* __restrict__ tileOffset,
                                                          const int4* __restrict__ meta,
                                                          const int* __restrict__ tileLevel,
                                                          const int* __restrict__ tileStart, int P, int ringBytes,
                                                          int metaLevels, uint32_t sliceBytes, bool dilu,
                                                          SPro<W> pro, W* __restrict__ y, int* errFlag,
                                                          bool pairRows) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int w = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
  const int T = static_cast<int>(blockIdx.x) * static_cast<int>(blockDim.x >> 5) + w;
  if (T >= P) return;  // the whole warp
  const KState* st = pro.st;
  if (st && st->done) return;
  unsigned char* my = smem + static_cast<size_t>(w) * sliceBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(my);
  int4* mt = reinterpret_cast<int4*>(my + 8 * kRingBarriers);
  unsigned char* ring = my + 8 * kRingBarriers + 16 * metaLevels;
  W* xs = reinterpret_cast<W*>(ring + ringBytes);
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  const int lv0 = tileLevel[T];
  const int L = tileLevel[T + 1] - lv0;
  const unsigned char* g = stream + tileOffset[T];
  for (int i = lane; i < L; i += 32) mt[i] = __ldg(meta + lv0 + i);
  if (lane == 0) {
    for (int i = 0; i < kRingBarriers; ++i) mbarInit(smemAddr(full + i), 1);
    fenceBarrierInit();
  }
  __syncwarp();
  // Lane 0: the copies of every level j with issueAfter(j) <= done (in
  // order; issueAfter never decreases along the levels).
  int issued = 0;
  uint32_t src = 0;
  auto issueUpTo = [&](int done) {
    while (issued < L) {
      const int4 m = mt[issued];
      if (RingLevelCode::issueAfter(m) > done) break;
      const uint32_t bytes = RingLevelCode::bytes(m);
      const uint32_t bar = smemAddr(full + issued % kRingBarriers);
      mbarExpectTx(bar, bytes);
      bulkLoad(smemAddr(ring + RingLevelCode::ringOffset(m)), g + src, bytes, bar);
      src += bytes;
      ++issued;
    }
  };
  if (lane == 0) issueUpTo(-1);
  {
    W beta = W(0), omega = W(0), alpha = W(0);
    bool first = true;
    if (st) {
      beta = cvt<W>(st->beta);
      omega = cvt<W>(st->omega);
      alpha = cvt<W>(st->alpha);
      first = st->iter == 0;
    }
    constexpr int kRows = sizeof(W) == 4 ? 16 : 8;
    for (int i0 = lane; i0 < nRows; i0 += 32 * kRows) {
      W v[kRows];
      pro.template rows<kRows>(base + i0, 32, base + nRows, beta, omega, alpha, first, v);
#pragma unroll
      for (int j = 0; j < kRows; ++j)
        if (i0 + j * 32 < nRows) xs[i0 + j * 32] = v[j];
    }
    if (lane == 0) xs[nRows] = W(0);
  }
  __syncwarp();
  int l = 0;
  bool bad = false;
  for (; l < L; ++l) {
    bad = !mbarWaitBounded(smemAddr(full + l % kRingBarriers), (l / kRingBarriers) & 1);
    if (__any_sync(0xFFFFFFFFu, bad)) break;
    const RingLevel<MV, COMPACT> cur = ringLevelAt<MV, COMPACT>(mt[l], ring);
    iluLevelRows<32>(cur, lane, nRows, dilu, pairRows, xs);
    __syncwarp();
    if (lane == 0) issueUpTo(l);
  }
  if (l < L) {
    if (lane == 0) {
      atomicExch(errFlag, GR_ETIMEOUT);
      // Let the copies still in flight land before the slice is released
      // (bounded): levels l .. issued - 1.
      for (int j = l; j < issued; ++j) mbarWaitBounded(smemAddr(full + j % kRingBarriers), (j / kRingBarriers) & 1);
    }
    return;
  }
  for (int i = lane; i < nRows; i += 32) y[base + i] = xs[i];
}

// Level l's rows of a Gauss-Seidel sweep for thread t of `stride` threads
// (gsRingKernel's compute warps' operations, in the same order). PAIR: a
// thread takes rows q and q + STRIDE together, both rows' loads before
// either's arithmetic and stores (rows of one level never read each other),
// so a level of up to 2 * STRIDE rows costs one dependent chain, not two.
template <int STRIDE, bool PAIR, class MV, class X, class W, bool COMPACT>
__device__ __forceinline__ void gsLevelRows(const RingLevel<MV, COMPACT>& cur, int t, bool seedB, const W* rhs,
                                            W* xs) {
  constexpr int kStep = PAIR ? 2 * STRIDE : STRIDE;
  if (cur.rec) {
    for (int q = t; q < cur.k; q += kStep) {
      const RowRecord r = ringRecord(cur, q, true);
      if (PAIR && q + STRIDE < cur.k) {
        const RowRecord r2 = ringRecord(cur, q + STRIDE, true);
        const W d = cvt<W>(r.inv), d2 = cvt<W>(r2.inv);
        const W s1 = recordDot(seedB ? rhs[r.row] : d, r, xs);
        const W s2 = recordDot(seedB ? rhs[r2.row] : d2, r2, xs);
        xs[r.row] = storeRound<X>(dvd(s1, d));
        xs[r2.row] = storeRound<X>(dvd(s2, d2));
      } else {
        const W d = cvt<W>(r.inv);
        const W sum = recordDot(seedB ? rhs[r.row] : d, r, xs);
        xs[r.row] = storeRound<X>(dvd(sum, d));
      }
    }
    return;
  }
  if (cur.E <= 8) {
    // Every entry's slot and value first, then the x values, then the sums
    // in order: the loads overlap.
    for (int q = t; q < cur.k; q += kStep) {
      constexpr int kR = PAIR ? 2 : 1;
      int il[kR], c[kR][8];
      MV v[kR][8];
      W d[kR], sum[kR], xv[kR][8];
      bool on[kR];
#pragma unroll
      for (int u = 0; u < kR; ++u) {
        const int qq = q + u * STRIDE;
        on[u] = u == 0 || qq < cur.k;
        if (on[u]) {
          il[u] = cur.row(qq);
          d[u] = cvt<W>(cur.invDiag(qq));
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (e < cur.E) cur.entry(e, qq, c[u][e], v[u][e]);
        }
      }
#pragma unroll
      for (int u = 0; u < kR; ++u)
        if (on[u]) {
          sum[u] = seedB ? rhs[il[u]] : d[u];
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (e < cur.E) xv[u][e] = xs[c[u][e]];
        }
#pragma unroll
      for (int u = 0; u < kR; ++u)
        if (on[u]) {
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (e < cur.E) sum[u] = sub(sum[u], mul(cvt<W>(v[u][e]), xv[u][e]));
        }
#pragma unroll
      for (int u = 0; u < kR; ++u)
        if (on[u]) xs[il[u]] = storeRound<X>(dvd(sum[u], d[u]));
    }
    return;
  }
  for (int q = t; q < cur.k; q += STRIDE) {
    const int il = cur.row(q);
    const W d = cvt<W>(cur.invDiag(q));
    W sum = seedB ? rhs[il] : d;
    for (int e = 0; e < cur.E; ++e) {
      int c;
      MV v;
      cur.entry(e, q, c, v);
      sum = sub(sum, mul(cvt<W>(v), xs[c]));
    }
    xs[il] = storeRound<X>(dvd(sum, d));
  }
}

// One Gauss-Seidel sweep with one warp per tile: gsRingKernel's sweep in
// iluWarpRingKernel's organisation (a shared-memory slice per warp, the
// warp's own barriers, __syncwarp between levels, lane 0 issuing its
// tile's copies).
template <class MV, class X, class W, bool COMPACT>
__global__ void __launch_bounds__(256) gsWarpRingKernel(
    const unsigned char* __restrict__ stream, const long long* __restrict__ tileOffset, const int4* __restrict__ meta,
    const int* __restrict__ tileLevel, const int* __restrict__ tileStart, const int* __restrict__ haloStart,
    const int* __restrict__ haloSrc, int P, int ringBytes, int metaLevels, uint32_t sliceBytes, bool seedB,
    SPro<X> pro, const X* __restrict__ xin, bool xinZero, X* __restrict__ xout, int* errFlag, bool inPlace,
    bool dropHalo, bool pairRows) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int w = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
  const int T = static_cast<int>(blockIdx.x) * static_cast<int>(blockDim.x >> 5) + w;
  if (T >= P) return;
  const KState* st = pro.st;
  if (st && st->done) return;
  unsigned char* my = smem + static_cast<size_t>(w) * sliceBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(my);
  int4* mt = reinterpret_cast<int4*>(my + 8 * kRingBarriers);
  unsigned char* ring = my + 8 * kRingBarriers + 16 * metaLevels;
  W* xs = reinterpret_cast<W*>(ring + ringBytes);
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  const int h0 = haloStart[T];
  const int nHalo = haloStart[T + 1] - h0;
  const int s0 = inPlace ? 0 : nRows;  // start values (in place: this sweep's slots)
  const int hb = s0 + nRows;           // halo
  W* rhs = xs + hb + nHalo + 1;
  const int lv0 = tileLevel[T];
  const int L = tileLevel[T + 1] - lv0;
  const unsigned char* g = stream + tileOffset[T];
  for (int i = lane; i < L; i += 32) mt[i] = __ldg(meta + lv0 + i);
  if (lane == 0) {
    for (int i = 0; i < kRingBarriers; ++i) mbarInit(smemAddr(full + i), 1);
    fenceBarrierInit();
  }
  __syncwarp();
  int issued = 0;
  uint32_t src = 0;
  // issueAfter of the next level to copy, kept in a register (levels never
  // issued: INT_MAX), so a level with nothing to issue costs one compare.
  int nextAfter = L > 0 ? RingLevelCode::issueAfter(mt[0]) : INT_MAX;
  auto issueUpTo = [&](int done) {
    while (nextAfter <= done) {
      const int4 m = mt[issued];
      const uint32_t bytes = RingLevelCode::bytes(m);
      const uint32_t bar = smemAddr(full + issued % kRingBarriers);
      mbarExpectTx(bar, bytes);
      bulkLoad(smemAddr(ring + RingLevelCode::ringOffset(m)), g + src, bytes, bar);
      src += bytes;
      ++issued;
      nextAfter = issued < L ? RingLevelCode::issueAfter(mt[issued]) : INT_MAX;
    }
  };
  if (lane == 0) issueUpTo(-1);
  constexpr int kRows = sizeof(W) == 4 ? 16 : 8;
  {
    // The right-hand side (seedB, with the fused p / s update) and the start
    // values of kRows rows a lane at once, all loads before any store.
    const bool withRhs = seedB || pro.kind != static_cast<int>(Prologue::Plain);
    X beta = X(0), omega = X(0), alpha = X(0);
    bool first = true;
    if (withRhs && st) {
      beta = cvt<X>(st->beta);
      omega = cvt<X>(st->omega);
      alpha = cvt<X>(st->alpha);
      first = st->iter == 0;
    }
    for (int i0 = lane; i0 < nRows; i0 += 32 * kRows) {
      W xv[kRows];
#pragma unroll
      for (int j = 0; j < kRows; ++j)
        xv[j] = !xinZero && i0 + j * 32 < nRows ? cvt<W>(xin[base + i0 + j * 32]) : W(0);
      if (withRhs) {
        X v[kRows];
        pro.template rows<kRows>(base + i0, 32, base + nRows, beta, omega, alpha, first, v);
        if (seedB) {
#pragma unroll
          for (int j = 0; j < kRows; ++j)
            if (i0 + j * 32 < nRows) rhs[i0 + j * 32] = cvt<W>(v[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < kRows; ++j)
        if (i0 + j * 32 < nRows) xs[s0 + i0 + j * 32] = xv[j];
    }
    // Halo cells: kRows source indices a lane, then their values.
    if (xinZero || dropHalo) {
      for (int h = lane; h < nHalo; h += 32) xs[hb + h] = W(0);
    } else {
      for (int h = lane; h < nHalo; h += 32 * kRows) {
        int src[kRows];
#pragma unroll
        for (int j = 0; j < kRows; ++j) src[j] = h + j * 32 < nHalo ? haloSrc[h0 + h + j * 32] : -1;
        W hv[kRows];
#pragma unroll
        for (int j = 0; j < kRows; ++j) hv[j] = src[j] >= 0 ? cvt<W>(xin[src[j]]) : W(0);
#pragma unroll
        for (int j = 0; j < kRows; ++j)
          if (src[j] >= 0) xs[hb + h + j * 32] = hv[j];
      }
    }
  }
  if (lane == 0) xs[hb + nHalo] = W(0);
  __syncwarp();
  int l = 0;
  bool bad = false;
  // The next level's table entry is decoded before the wait for its block.
  RingLevel<MV, COMPACT> nxt = ringLevelAt<MV, COMPACT>(L > 0 ? mt[0] : make_int4(0, 0, 0, 0), ring);
  for (; l < L; ++l) {
    const RingLevel<MV, COMPACT> cur = nxt;
    if (l + 1 < L) nxt = ringLevelAt<MV, COMPACT>(mt[l + 1], ring);
    bad = !mbarWaitBounded(smemAddr(full + l % kRingBarriers), (l / kRingBarriers) & 1);
    if (__any_sync(0xFFFFFFFFu, bad)) break;
    if (pairRows) gsLevelRows<32, true, MV, X, W, COMPACT>(cur, lane, seedB, rhs, xs);
    else gsLevelRows<32, false, MV, X, W, COMPACT>(cur, lane, seedB, rhs, xs);
    __syncwarp();
    if (lane == 0) issueUpTo(l);
  }
  if (l < L) {
    if (lane == 0) {
      atomicExch(errFlag, GR_ETIMEOUT);
      for (int j = l; j < issued; ++j) mbarWaitBounded(smemAddr(full + j % kRingBarriers), (j / kRingBarriers) & 1);
    }
    return;
  }
  for (int i = lane; i < nRows; i += 32) xout[base + i] = cvt<X>(xs[i]);
}

}  // namespace dev

// ---------------------------------------------------------------------------
size_t iluRingSmem(const DeviceMatrix& A, const LevelRing& R, DType W) {
  (void)A;
  return static_cast<size_t>(ringFixedSmemSlots(R.maxTileLevels, R.maxXSlots, static_cast<i64>(dtypeSize(W))) +
                             R.ringBytes);
}

void launchRingPack(DeviceMatrix& A, const LevelRing& R, void* stream, const void* F, const void* inv,
                    cudaStream_t s) {
  launchPackBytes(A, R.templ.get(), R.bytes, R.valPos.as<int>(), R.valSrc.as<int>(), R.nVal, R.invPos.as<int>(),
                  R.invSrc.as<int>(), R.nInv, stream, F, inv, s);
}

namespace {
template <class MV, class W, int CW, bool WAITER = true, bool PRODUCER = true>
auto ringKernelFor(bool compact, bool unroll) {
  return compact ? (unroll ? dev::iluRingKernel<MV, W, true, true, CW, WAITER, PRODUCER>
                           : dev::iluRingKernel<MV, W, false, true, CW, WAITER, PRODUCER>)
                 : (unroll ? dev::iluRingKernel<MV, W, true, false, CW, WAITER, PRODUCER>
                           : dev::iluRingKernel<MV, W, false, false, CW, WAITER, PRODUCER>);
}

template <class MV, class W>
void ringApplyT(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& p, void* y,
                int l2Ahead, bool unroll, bool pairRows, cudaStream_t s, int computeWarps, bool waiter,
                bool producer) {
  const size_t smem = iluRingSmem(A, R, dtypeOf<W>());
  if (computeWarps != 0 && computeWarps != 1 && computeWarps != 2 && computeWarps != 4 && computeWarps != 8)
    fail(GR_EINVAL, "computeWarps must be 1, 2, 4 or 8 (0: the default)");
  if (!waiter && computeWarps != 0) fail(GR_EINVAL, "waitingWarp false needs the default computeWarps");
  if (!waiter && !producer) fail(GR_EINVAL, "producerWarp false needs the waiting warp");
  if (!producer && computeWarps != 0 && computeWarps != 4)
    fail(GR_EINVAL, "producerWarp false runs with the default computeWarps or 4");
  auto kernel = !waiter             ? ringKernelFor<MV, W, 0, false>(R.compact, unroll)
                : !producer         ? (computeWarps == 4 ? ringKernelFor<MV, W, 4, true, false>(R.compact, unroll)
                                                         : ringKernelFor<MV, W, 0, true, false>(R.compact, unroll))
                : computeWarps == 1 ? ringKernelFor<MV, W, 1>(R.compact, unroll)
                : computeWarps == 2 ? ringKernelFor<MV, W, 2>(R.compact, unroll)
                : computeWarps == 4 ? ringKernelFor<MV, W, 4>(R.compact, unroll)
                : computeWarps == 8 ? ringKernelFor<MV, W, 8>(R.compact, unroll)
                                    : ringKernelFor<MV, W, 0>(R.compact, unroll);
  const int threads =
      (computeWarps > 0 ? 32 * computeWarps : dev::RingShape<W>::compute) + (waiter ? 32 : 0) + (producer ? 32 : 0);
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
  preferSharedCarveout(reinterpret_cast<const void*>(kernel));
  if (p.stIndex && R.group != 1) fail(GR_EUNSUPPORTED, "batched solves run one tile per block");
  dev::SPro<W> pro{static_cast<int>(p.kind), static_cast<const W*>(p.b), static_cast<const W*>(p.r),
                   static_cast<W*>(p.pOrS), static_cast<const W*>(p.v), p.st, p.stIndex};
  kernel<<<R.numGroups, threads, smem, s>>>(static_cast<const unsigned char*>(stream),
                                             R.tileOffset.as<long long>(), R.meta.as<int4>(), R.tileLevel.as<int>(),
                                             R.groupStart.as<int>(),
                                             static_cast<int>(R.ringBytes), R.maxTileLevels,
                                             static_cast<uint32_t>(l2Ahead < 0 ? dev::kPrefetchAhead : l2Ahead) & ~15u, dilu, pro,
                                             static_cast<W*>(y), A.errFlag.as<int>(), pairRows);
  checkLaunch("ilu_ring");
}
}  // namespace

int iluRingBlocksPerSM(const DeviceMatrix& A, const LevelRing& R, DType W, int computeWarps) {
  const size_t smem = iluRingSmem(A, R, W);
  const void* fn = nullptr;
  int threads = 0;
  if (W == DType::F32) {
    fn = reinterpret_cast<const void*>(computeWarps == 4 ? ringKernelFor<float, float, 4>(R.compact, true)
                                                         : ringKernelFor<float, float, 0>(R.compact, true));
    threads = (computeWarps == 4 ? 128 : dev::RingShape<float>::compute) + 64;
  } else {
    fn = reinterpret_cast<const void*>(computeWarps == 4 ? ringKernelFor<double, double, 4>(R.compact, true)
                                                         : ringKernelFor<double, double, 0>(R.compact, true));
    threads = (computeWarps == 4 ? 128 : dev::RingShape<double>::compute) + 64;
  }
  ensureDynamicSmem(fn, smem);
  preferSharedCarveout(fn);
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

int ringBlocksPerSMWithoutSmem(DType vt, RingKind kind) {
  int n = 0;
  const bool gs = kind != RingKind::Ilu;
  const void* fn = vt == DType::F64
                       ? (gs ? reinterpret_cast<const void*>(dev::gsRingKernel<double, double, double, true>)
                             : reinterpret_cast<const void*>(dev::iluRingKernel<double, double, true, true>))
                       : (gs ? reinterpret_cast<const void*>(dev::gsRingKernel<float, float, float, true>)
                             : reinterpret_cast<const void*>(dev::iluRingKernel<float, float, true, true>));
  const int threads = vt == DType::F64 ? dev::RingShape<double>::threads : dev::RingShape<float>::threads;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

namespace {
inline size_t gsWarpRingSlice(const LevelRing& R, DType W) {
  const size_t b = 8 * kRingBarriers + 16 * static_cast<size_t>(R.maxTileLevels) + static_cast<size_t>(R.ringBytes) +
                   static_cast<size_t>(R.maxXSlots) * dtypeSize(W);
  return (b + 127) / 128 * 128;
}
template <class MV, class X, class W>
void gsRingT(DeviceMatrix& A, const LevelRing& R, const void* stream, const PrologueArgs& p, bool seedB,
             const void* xin, bool xinZero, void* xout, int warps, cudaStream_t s, bool dropHalo, bool pairRows) {
  if (R.kind == RingKind::Ilu) fail(GR_EINVAL, "not a Gauss-Seidel ring");
  if (R.kind == RingKind::GaussSeidelLower && !xinZero)
    fail(GR_EINVAL, "a lower-only Gauss-Seidel ring sweeps from x = 0 only");
  if (warps > 0) {
    if (warps > 8) fail(GR_EINVAL, "warpsPerBlock must be 1..8");
    if (p.stIndex) fail(GR_EUNSUPPORTED, "batched solves use the block ring kernel");
    const size_t slice = gsWarpRingSlice(R, dtypeOf<W>());
    const size_t smem = slice * static_cast<size_t>(warps);
    auto kernel = R.compact ? dev::gsWarpRingKernel<MV, X, W, true> : dev::gsWarpRingKernel<MV, X, W, false>;
    ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
    preferSharedCarveout(reinterpret_cast<const void*>(kernel));
    dev::SPro<X> pro{static_cast<int>(p.kind), static_cast<const X*>(p.b), static_cast<const X*>(p.r),
                     static_cast<X*>(p.pOrS), static_cast<const X*>(p.v), p.st, nullptr};
    kernel<<<(R.numGroups + warps - 1) / warps, 32 * warps, smem, s>>>(
        static_cast<const unsigned char*>(stream), R.tileOffset.as<long long>(), R.meta.as<int4>(),
        R.tileLevel.as<int>(), R.groupStart.as<int>(), R.haloStart.as<int>(), R.haloSrc.as<int>(), R.numGroups,
        static_cast<int>(R.ringBytes), R.maxTileLevels, static_cast<uint32_t>(slice), seedB, pro,
        static_cast<const X*>(xin), xinZero, static_cast<X*>(xout), A.errFlag.as<int>(), R.gsInPlace, dropHalo,
        pairRows);
    checkLaunch("gs_warp_ring");
    return;
  }
  const size_t smem = iluRingSmem(A, R, dtypeOf<W>());
  auto kernel = R.compact ? dev::gsRingKernel<MV, X, W, true> : dev::gsRingKernel<MV, X, W, false>;
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
  preferSharedCarveout(reinterpret_cast<const void*>(kernel));
  // Batches: the state of tile T's system is st[stIndex[T]].
  dev::SPro<X> pro{static_cast<int>(p.kind), static_cast<const X*>(p.b), static_cast<const X*>(p.r),
                   static_cast<X*>(p.pOrS), static_cast<const X*>(p.v), p.st, p.stIndex};
  kernel<<<R.numGroups, dev::RingShape<W>::threads, smem, s>>>(
      static_cast<const unsigned char*>(stream), R.tileOffset.as<long long>(), R.meta.as<int4>(),
      R.tileLevel.as<int>(), R.groupStart.as<int>(), R.haloStart.as<int>(), R.haloSrc.as<int>(),
      static_cast<int>(R.ringBytes), R.maxTileLevels, seedB, pro, static_cast<const X*>(xin), xinZero,
      static_cast<X*>(xout), A.errFlag.as<int>(), R.gsInPlace, dropHalo);
  checkLaunch("gs_ring");
}
}  // namespace

size_t gsWarpRingSmem(const LevelRing& R, DType W, int warpsPerBlock) {
  return gsWarpRingSlice(R, W) * static_cast<size_t>(warpsPerBlock);
}

void launchGsRing(DeviceMatrix& A, const LevelRing& R, const void* stream, const PrologueArgs& pro, bool seedB,
                  const void* xin, bool xinZero, void* xout, DType X, DType W, cudaStream_t s, int warps, bool dropHalo,
                  bool pairRows) {
  if (A.vt == DType::F32 && X == DType::F32 && W == DType::F32)
    gsRingT<float, float, float>(A, R, stream, pro, seedB, xin, xinZero, xout, warps, s, dropHalo, pairRows);
  else if (A.vt == DType::F32 && X == DType::F32 && W == DType::F64)
    gsRingT<float, float, double>(A, R, stream, pro, seedB, xin, xinZero, xout, warps, s, dropHalo, pairRows);
  else if (A.vt == DType::F32 && X == DType::F64 && W == DType::F64)
    gsRingT<float, double, double>(A, R, stream, pro, seedB, xin, xinZero, xout, warps, s, dropHalo, pairRows);
  else if (A.vt == DType::F64 && X == DType::F64 && W == DType::F64)
    gsRingT<double, double, double>(A, R, stream, pro, seedB, xin, xinZero, xout, warps, s, dropHalo, pairRows);
  else
    fail(GR_EUNSUPPORTED, "Gauss-Seidel: float64 coefficients need float64 vectors, and the working type must be "
                          "the vectors' type or float64 over float32 vectors");
}

namespace {
inline size_t warpRingSlice(const LevelRing& R, DType W) {
  const size_t b = 8 * kRingBarriers + 16 * static_cast<size_t>(R.maxTileLevels) + static_cast<size_t>(R.ringBytes) +
                   static_cast<size_t>(R.maxGroupRows + 1) * dtypeSize(W);
  return (b + 127) / 128 * 128;
}
template <class MV, class W>
void warpRingT(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& p, void* y,
               int warpsPerBlock, bool pairRows, cudaStream_t s) {
  if (R.kind != RingKind::Ilu || R.group != 1) fail(GR_EINVAL, "the warp ring kernel runs one tile per warp");
  if (p.stIndex) fail(GR_EUNSUPPORTED, "batched solves use the block ring kernel");
  const size_t slice = warpRingSlice(R, dtypeOf<W>());
  const size_t smem = slice * static_cast<size_t>(warpsPerBlock);
  auto kernel = R.compact ? dev::iluWarpRingKernel<MV, W, true> : dev::iluWarpRingKernel<MV, W, false>;
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), smem);
  preferSharedCarveout(reinterpret_cast<const void*>(kernel));
  dev::SPro<W> pro{static_cast<int>(p.kind), static_cast<const W*>(p.b), static_cast<const W*>(p.r),
                   static_cast<W*>(p.pOrS), static_cast<const W*>(p.v), p.st, nullptr};
  const int blocks = (R.numGroups + warpsPerBlock - 1) / warpsPerBlock;
  kernel<<<blocks, 32 * warpsPerBlock, smem, s>>>(
      static_cast<const unsigned char*>(stream), R.tileOffset.as<long long>(), R.meta.as<int4>(), R.tileLevel.as<int>(),
      R.groupStart.as<int>(), R.numGroups, static_cast<int>(R.ringBytes), R.maxTileLevels,
      static_cast<uint32_t>(slice), dilu, pro, static_cast<W*>(y), A.errFlag.as<int>(), pairRows);
  checkLaunch("ilu_warp_ring");
}
}  // namespace

size_t iluWarpRingSmem(const LevelRing& R, DType W, int warpsPerBlock) {
  return warpRingSlice(R, W) * static_cast<size_t>(warpsPerBlock);
}

void launchIluWarpRing(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& pro,
                       void* y, DType W, int warpsPerBlock, bool pairRows, cudaStream_t s) {
  if (warpsPerBlock < 1 || warpsPerBlock > 8) fail(GR_EINVAL, "warpsPerBlock must be 1..8");
  if (A.vt == DType::F32 && W == DType::F32)
    warpRingT<float, float>(A, R, stream, dilu, pro, y, warpsPerBlock, pairRows, s);
  else if (A.vt == DType::F32 && W == DType::F64)
    warpRingT<float, double>(A, R, stream, dilu, pro, y, warpsPerBlock, pairRows, s);
  else if (A.vt == DType::F64 && W == DType::F64)
    warpRingT<double, double>(A, R, stream, dilu, pro, y, warpsPerBlock, pairRows, s);
  else fail(GR_EUNSUPPORTED, "ILU apply with float64 coefficients and float32 vectors");
}

void launchIluRing(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& pro,
                   void* y, DType W, int l2Ahead, bool unroll, cudaStream_t s, bool pairRows, int computeWarps,
                   bool waiter, bool producer) {
  if (A.vt == DType::F32 && W == DType::F32)
    ringApplyT<float, float>(A, R, stream, dilu, pro, y, l2Ahead, unroll, pairRows, s, computeWarps, waiter,
                             producer);
  else if (A.vt == DType::F32 && W == DType::F64)
    ringApplyT<float, double>(A, R, stream, dilu, pro, y, l2Ahead, unroll, pairRows, s, computeWarps, waiter,
                              producer);
  else if (A.vt == DType::F64 && W == DType::F64)
    ringApplyT<double, double>(A, R, stream, dilu, pro, y, l2Ahead, unroll, pairRows, s, computeWarps, waiter,
                               producer);
  else fail(GR_EUNSUPPORTED, "ILU apply with float64 coefficients and float32 vectors");
}

}  // namespace gr

// Device matrix set-up and the SpMV / residual / norm kernels.
//
// SpMV and residual follow CRSMatrix::spmv / CRSMatrix::residual
// (matrix/details/crs/CRSMatrix.cpp:42-128): per row, the diagonal product
// first, then the off-diagonal products added in tile-local column order,
// each operation rounded in the intermediate type. The reference's halo
// exchange (MatrixBase.cpp:36-109) becomes a direct read of the neighbour
// tile's entry of x, which is the value the exchange would have copied.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <set>
#include <mutex>

#include "device.hpp"
#include "devmath.cuh"
#include "sell.cuh"

namespace gr {

namespace {
std::atomic<i64> g_launches{0};
thread_local bool g_capturing = false;
thread_local i64 g_captured = 0;
}

void noteLaunch(int count) {
  if (g_capturing) g_captured += count;
  else g_launches.fetch_add(count);
}
i64 capturedCount() { return g_captured; }
i64 launchCount() { return g_launches.load(); }
void setCapturing(bool on) { g_capturing = on; }
bool capturing() { return g_capturing; }

void cudaCheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? GR_ENOMEM : GR_ECUDA;
    fail(code, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
  }
}

// Device memory comes from the device's stream-ordered pool. cudaFree may
// wait for all work on the device, which would serialise solves running
// concurrently on other streams; cudaFreeAsync does not. Freed blocks stay
// in the process's pool (release threshold raised once per device) and are
// reused by later allocations.
namespace {
std::once_flag g_poolOnce[64];

void keepPoolMemory() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::call_once(g_poolOnce[dev], [dev] {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  });
}
}  // namespace

void ensureDynamicSmem(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return;  // within the default limit
  int dev = 0;
  GR_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> raised;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = raised[{dev, fn}];
  if (bytes <= cur) return;
  GR_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
  cur = bytes;
}

void preferSharedCarveout(const void* fn) {
  int dev = 0;
  GR_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  std::lock_guard<std::mutex> lock(mu);
  if (!done.insert({dev, fn}).second) return;
  GR_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
}

namespace {
// Device blocks released by DBufs, kept for reuse (by device and size, up to
// kBlockCacheBytes in all). A solver's setup then takes its buffers from here
// rather than from the stream-ordered allocator, whose requests for memory it
// had to grow for took up to a quarter of a second on B200. Every owner
// synchronises the buffer's stream before releasing it, so a cached block has
// no work pending.
struct BlockCache {
  std::mutex mu;
  std::multimap<std::pair<int, size_t>, void*> blocks;
  size_t bytes = 0;
};
BlockCache& blockCache() {
  static BlockCache* c = new BlockCache();  // outlives every DBuf
  return *c;
}
constexpr size_t kBlockCacheBytes = size_t(8) << 30;

// Returns every cached block of `dev` to the allocator.
void trimBlockCache(int dev) {
  BlockCache& c = blockCache();
  std::lock_guard<std::mutex> lock(c.mu);
  for (auto it = c.blocks.begin(); it != c.blocks.end();) {
    if (it->first.first == dev) {
      cudaFreeAsync(it->second, cudaStreamPerThread);
      c.bytes -= it->first.second;
      it = c.blocks.erase(it);
    } else {
      ++it;
    }
  }
  cudaStreamSynchronize(cudaStreamPerThread);
}
}  // namespace

void DBuf::alloc(size_t bytes) {
  release();
  if (bytes == 0) bytes = 1;
  int dev = 0;
  GR_CUDA(cudaGetDevice(&dev));
  {
    // A cached block of this device at most 1/8 larger than asked for.
    BlockCache& c = blockCache();
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.blocks.lower_bound({dev, bytes});
    if (it != c.blocks.end() && it->first.first == dev && it->first.second <= bytes + bytes / 8) {
      p_ = it->second;
      bytes_ = it->first.second;
      dev_ = dev;
      c.bytes -= bytes_;
      c.blocks.erase(it);
      return;
    }
  }
  keepPoolMemory();
  cudaError_t e = cudaMallocAsync(&p_, bytes, cudaStreamPerThread);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
  if (e == cudaErrorMemoryAllocation) {
    // Out of memory: give the cached blocks back and try once more.
    (void)cudaGetLastError();
    trimBlockCache(dev);
    e = cudaMallocAsync(&p_, bytes, cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
  }
  if (e != cudaSuccess) {
    p_ = nullptr;
    (void)cudaGetLastError();
    fail(GR_ENOMEM, "allocation of " + std::to_string(bytes) + " device bytes failed: " +
                        cudaGetErrorString(e));
  }
  bytes_ = bytes;
  dev_ = dev;
}

// The owner guarantees that no work using the buffer is still pending (it
// synchronises the stream the buffer was used on before releasing it).
void DBuf::release() {
  if (!p_) return;
  {
    BlockCache& c = blockCache();
    std::lock_guard<std::mutex> lock(c.mu);
    if (c.bytes + bytes_ <= kBlockCacheBytes) {
      c.blocks.insert({{dev_, bytes_}, p_});
      c.bytes += bytes_;
      p_ = nullptr;
      bytes_ = 0;
      return;
    }
  }
  cudaFreeAsync(p_, cudaStreamPerThread);
  p_ = nullptr;
  bytes_ = 0;
}

void uploadValues(DBuf& dst, const std::vector<double>& v, DType t) {
  if (t == DType::F64) {
    dst.upload(v);
  } else if (t == DType::F32) {
    std::vector<float> f(v.size());
    parallelChunks(static_cast<i64>(v.size()), [&](i64 b, i64 e) {
      for (i64 i = b; i < e; ++i) f[i] = static_cast<float>(v[i]);
    });
    dst.upload(f);
  } else {
    fail(GR_EUNSUPPORTED, "coefficient type must be float32 or float64");
  }
}

// ---------------------------------------------------------------------------
// SELL layout on the host.
SellHost buildSell(const HostMatrix& H, int layout) {
  if (layout < -1 || layout > 1) fail(GR_EINVAL, "spmv layout must be -1, 0 or 1");
  SellHost S;
  const i64 n = H.n;
  const i64 nChunks = (n + 31) / 32;
  std::vector<i64> chunkLen(nChunks, 0);
  parallelChunks(nChunks, [&](i64 b, i64 e) {
    for (i64 c = b; c < e; ++c) {
      i64 mx = 0;
      for (i64 r = c * 32; r < std::min<i64>(n, c * 32 + 32); ++r) mx = std::max(mx, H.rowPtr[r + 1] - H.rowPtr[r]);
      chunkLen[c] = mx;
    }
  });
  S.base.assign(nChunks + 1, 0);
  i64 acc = 0;
  for (i64 c = 0; c < nChunks; ++c) {
    S.base[c] = static_cast<i32>(acc);
    acc += 32 * chunkLen[c];
    if (acc >= (i64(1) << 31)) fail(GR_EUNSUPPORTED, "SELL storage exceeds 2^31 slots");
  }
  S.base[nChunks] = static_cast<i32>(acc);
  S.slots = acc;
  S.col.assign(acc, -1);
  S.val.assign(acc, 0.0);
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e; ++r) {
      i64 c = r / 32, lane = r % 32;
      // Slot k holds the row's k-th term of its summation order: local
      // column order for CRS, the LDU order (sumRank) for LDU matrices.
      for (i64 k = 0; k < H.rowPtr[r + 1] - H.rowPtr[r]; ++k) {
        const i64 p = H.rowPtr[r] + k;
        const i64 slot = H.sumRank.empty() ? k : H.sumRank[p];
        i64 s = S.base[c] + 32 * slot + lane;
        S.col[s] = H.colPerm[p];
        S.val[s] = H.offDiag[p];
      }
    }
  });
  // Automatic: 32-bit columns. On B200 the 16-bit walk (two loads, a vote
  // and a shuffle a slot) ran the 192^3 SpMV in 104.6 us against 78.1 us
  // for the 32-bit layout, despite moving a quarter fewer bytes.
  if (layout <= 0) return S;
  // 16-bit offsets; far entries counted per chunk in slot order.
  std::vector<int16_t> d16(acc, static_cast<int16_t>(dev::kSellPad));
  std::vector<i32> farCount(nChunks + 1, 0);
  parallelChunks(nChunks, [&](i64 b, i64 e) {
    for (i64 c = b; c < e; ++c) {
      i32 f = 0;
      for (i64 s = S.base[c]; s < S.base[c + 1]; ++s) {
        if (S.col[s] < 0) continue;
        const i64 row = c * 32 + (s - S.base[c]) % 32;
        const i64 d = static_cast<i64>(S.col[s]) - row;
        if (d == 0 || d < -32767 || d > 32767) {
          d16[s] = static_cast<int16_t>(dev::kSellFar);
          ++f;
        } else {
          d16[s] = static_cast<int16_t>(d);
        }
      }
      farCount[c] = f;
    }
  });
  i64 far = 0, maxFar = 0;
  for (i64 c = 0; c < nChunks; ++c) {
    far += farCount[c];
    maxFar = std::max<i64>(maxFar, farCount[c]);
  }
  S.maxChunkFar = maxFar;
  // The device hands a chunk's far columns out of two registers of the
  // warp's 32 lanes.
  if (maxFar > dev::kSellMaxFar)
    fail(GR_EUNSUPPORTED, "the 16-bit SpMV layout needs at most " + std::to_string(dev::kSellMaxFar) +
                              " far columns per chunk of 32 rows (this matrix has " + std::to_string(maxFar) + ")");

  S.compact = true;
  S.d16 = std::move(d16);
  S.farBase.assign(nChunks + 1, 0);
  i64 run = 0;
  for (i64 c = 0; c < nChunks; ++c) {
    S.farBase[c] = static_cast<i32>(run);
    run += farCount[c];
  }
  S.farBase[nChunks] = static_cast<i32>(run);
  S.farCol.resize(run);
  parallelChunks(nChunks, [&](i64 b, i64 e) {
    for (i64 c = b; c < e; ++c) {
      i32 f = S.farBase[c];
      for (i64 s = S.base[c]; s < S.base[c + 1]; ++s)
        if (S.d16[s] == dev::kSellFar) S.farCol[f++] = S.col[s];
    }
  });
  return S;
}

void checkSellDecode(const SellHost& S, i64 n) {
  if (!S.compact) return;
  const i64 nChunks = (n + 31) / 32;
  for (i64 c = 0; c < nChunks; ++c) {
    const i64 s0 = S.base[c];
    const i64 K = (S.base[c + 1] - s0) / 32;
    i64 run = 0;  // the warp's running count of far slots, votes in k order
    for (i64 k = 0; k < K; ++k) {
      i64 below = 0;  // far slots of lower lanes at this k
      for (i64 lane = 0; lane < 32; ++lane) {
        const i64 s = s0 + 32 * k + lane;
        const int d = S.d16[s];
        i64 colv;
        if (d == dev::kSellPad) {
          colv = -1;
        } else if (d == dev::kSellFar) {
          const i64 idx = S.farBase[c] + run + below;
          if (idx >= S.farBase[c + 1]) fail(GR_EINVAL, "SELL far list overrun in chunk " + std::to_string(c));
          colv = S.farCol[idx];
          ++below;
        } else {
          colv = c * 32 + lane + d;
        }
        if (colv != S.col[s])
          fail(GR_EINVAL, "SELL 16-bit layout decodes slot " + std::to_string(s) + " to column " +
                              std::to_string(colv) + ", expected " + std::to_string(S.col[s]));
      }
      run += below;
    }
    if (S.farBase[c] + run != S.farBase[c + 1]) fail(GR_EINVAL, "SELL far count mismatch in chunk " + std::to_string(c));
  }
}

// ---------------------------------------------------------------------------
// Device matrix (HostMatrix::copyToTile, CRSHostMatrix.cpp:356-378).
DeviceMatrix::DeviceMatrix(std::shared_ptr<HostMatrix> h) : host(std::move(h)) {
  const HostMatrix& H = *host;
  GR_CUDA(cudaGetDevice(&device));
  GR_CUDA(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device));
  // A blocking stream: work on the legacy default stream (e.g. PyTorch's) and
  // on this stream stays ordered.
  GR_CUDA(cudaStreamCreateWithFlags(&ownStream, cudaStreamDefault));
  stream = ownStream;
  n = static_cast<i32>(H.n);
  m = H.m;
  P = H.P;
  vt = H.valueType;

  // Sliced ELLPACK, chunk height 32, rows in tile order.
  SellHost S = buildSell(H, H.spmvLayout);
  sell.n = n;
  sell.nChunks = (n + 31) / 32;
  sell.slots = S.slots;
  sell.compact = S.compact;
  sell.far = static_cast<i64>(S.farCol.size());
  sell.base.upload(S.base);
  if (S.compact) {
    sell.d16.upload(S.d16);
    std::vector<i32> fc = S.farCol;
    if (fc.empty()) fc.push_back(0);  // a valid pointer for the kernels
    sell.farCol.upload(fc);
    sell.farBase.upload(S.farBase);
    uploadValues(sell.val, S.val, vt);
  } else if (vt == DType::F32) {
    std::vector<int2> ent(S.slots);
    parallelChunks(S.slots, [&](i64 b, i64 e) {
      for (i64 s = b; s < e; ++s) {
        float f = static_cast<float>(S.val[s]);
        int bits;
        std::memcpy(&bits, &f, sizeof(bits));
        ent[s] = make_int2(S.col[s], bits);
      }
    });
    sell.ent.upload(ent);
  } else {
    sell.col.upload(S.col);
    uploadValues(sell.val, S.val, vt);
  }
  uploadValues(diag, H.diag, vt);
  std::vector<i32> ts(H.tileStart.begin(), H.tileStart.end());
  tileStart.upload(ts);
  iperm.upload(H.iperm);

  redBlocks = numSMs * 8;
  sellGridCap();  // the occupancy query outside any stream capture
  partials.alloc(sizeof(double) * redBlocks * 8);
  counter.alloc(sizeof(unsigned) * 16);
  GR_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(unsigned) * 16, ownStream));
  scalarOut.alloc(sizeof(double) * 8);
  errFlag.alloc(sizeof(int));
  GR_CUDA(cudaMemsetAsync(errFlag.get(), 0, sizeof(int), ownStream));
  // Only this matrix's stream: other solves may be running on the device.
  GR_CUDA(cudaStreamSynchronize(ownStream));
}

DeviceMatrix::~DeviceMatrix() {
  if (ownStream) {
    cudaStreamSynchronize(ownStream);
    cudaStreamDestroy(ownStream);
  }
}

void DeviceMatrix::makeBatch(const std::vector<i64>& rowBegin, const std::vector<i64>& rowReal,
                             const std::vector<i32>& tileBegin) {
  const int S = static_cast<int>(rowBegin.size());
  if (S < 1 || static_cast<int>(rowReal.size()) != S || static_cast<int>(tileBegin.size()) != S + 1)
    fail(GR_EINVAL, "batch tables");
  auto B = std::make_unique<BatchSeg>();
  B->systems = S;
  B->rowBegin = rowBegin;
  B->rowReal = rowReal;
  B->tileBegin = tileBegin;
  std::vector<i32> r0(S), r1(S);
  // Per system, the block counts a solve of that system alone would use
  // (spmvBlocks and the elementwise grid), so that the reductions combine the
  // same partials in the same order.
  std::vector<i32> cSys, cRank, cBlocks(S), cBlock0(S), eSys, eRank, eBlocks(S), eBlock0(S);
  for (int s = 0; s < S; ++s) {
    if (rowBegin[s] % 32 != 0) fail(GR_EINVAL, "batch systems must start at a multiple of 32 rows");
    r0[s] = static_cast<i32>(rowBegin[s]);
    r1[s] = static_cast<i32>(rowBegin[s] + rowReal[s]);
    const i64 chunks = (rowReal[s] + 31) / 32;
    cBlocks[s] = static_cast<i32>(std::max<i64>(1, std::min<i64>((chunks + 7) / 8, sellGridCap())));
    eBlocks[s] = static_cast<i32>(std::max<i64>(1, std::min<i64>(redBlocks, (rowReal[s] + 255) / 256)));
    cBlock0[s] = static_cast<i32>(cSys.size());
    eBlock0[s] = static_cast<i32>(eSys.size());
    for (int j = 0; j < cBlocks[s]; ++j) {
      cSys.push_back(s);
      cRank.push_back(j);
    }
    for (int j = 0; j < eBlocks[s]; ++j) {
      eSys.push_back(s);
      eRank.push_back(j);
    }
  }
  B->chunkGrid = static_cast<int>(cSys.size());
  B->elemGrid = static_cast<int>(eSys.size());
  B->row0.upload(r0);
  B->rowEnd.upload(r1);
  B->chunkSys.upload(cSys);
  B->chunkRank.upload(cRank);
  B->chunkBlocks.upload(cBlocks);
  B->chunkBlock0.upload(cBlock0);
  B->elemSys.upload(eSys);
  B->elemRank.upload(eRank);
  B->elemBlocks.upload(eBlocks);
  B->elemBlock0.upload(eBlock0);
  B->partials.alloc(sizeof(double) * 2 * std::max(B->chunkGrid, B->elemGrid));
  B->counters.alloc(sizeof(unsigned) * S);
  GR_CUDA(cudaMemsetAsync(B->counters.get(), 0, sizeof(unsigned) * S, ownStream));
  std::vector<i32> tileSys(P);
  for (int s = 0; s < S; ++s)
    for (i32 T = tileBegin[s]; T < tileBegin[s + 1]; ++T) tileSys[T] = s;
  B->tileSys.upload(tileSys);
  GR_CUDA(cudaStreamSynchronize(ownStream));
  batch = std::move(B);
}

int DeviceMatrix::sellGridCap() const {
  if (sellCap == 0) {
    // One wave: as many 256-thread blocks as the row-chunk Krylov kernels of
    // this value type and SELL layout keep resident on every SM.
    const int occ = sellKernelOccupancy(vt, sell.compact);
    sellCap = std::max(1, std::min(redBlocks, numSMs * std::max(1, occ)));
  }
  return sellCap;
}

int DeviceMatrix::spmvBlocks() const {
  int need = (sell.nChunks + 7) / 8;
  return std::max(1, std::min(need, sellGridCap()));
}

void DeviceMatrix::ensureLocalCrs() {
  if (haveLocalCrs) return;
  const HostMatrix& H = *host;
  std::vector<i32> rp(H.rowPtr.begin(), H.rowPtr.end());
  rowPtr.upload(rp);
  colLocal.upload(H.colLocal);
  uploadValues(offDiag, H.offDiag, vt);
  haveLocalCrs = true;
}

namespace dev {
// SELL value of every slot from the tile-local CRS values (padding: 0).
template <class MV>
__global__ void sellScatterKernel(const int* __restrict__ src, const MV* __restrict__ off, int2* ent, MV* val,
                                  long long slots) {
  for (long long s = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; s < slots;
       s += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int p = src[s];
    const MV v = p >= 0 ? off[p] : MV(0);
    if (ent) ent[s].y = __float_as_int(static_cast<float>(v));
    else val[s] = v;
  }
}
}  // namespace dev

namespace dev {
// New coefficients from global CRS values (FP64, natural order) gathered on
// the device: tile-local CRS off-diagonals, SELL slots (padding: 0) and the
// tile-ordered diagonal, each rounded once to the coefficient type.
template <class MV, class SRC>
__global__ void globalValuesKernel(const SRC* __restrict__ gVal, const SRC* __restrict__ gDiag,
                                   const int* __restrict__ srcOff, const int* __restrict__ srcSell,
                                   const int* __restrict__ iperm, MV* off, int2* ent, MV* val, MV* diag,
                                   long long m, long long slots, int n) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long i0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  for (long long p = i0; p < m; p += stride) off[p] = static_cast<MV>(gVal[srcOff[p]]);
  for (long long s = i0; s < slots; s += stride) {
    const int g = srcSell[s];
    const MV v = g >= 0 ? static_cast<MV>(gVal[g]) : MV(0);
    if (ent) ent[s].y = __float_as_int(static_cast<float>(v));
    else val[s] = v;
  }
  for (long long p = i0; p < n; p += stride) diag[p] = static_cast<MV>(gDiag[iperm[p]]);
}
}  // namespace dev

namespace {
// Values converted to t and copied into an existing device buffer.
void copyValuesInto(DBuf& dst, const std::vector<double>& v, DType t, cudaStream_t s) {
  const size_t bytes = v.size() * dtypeSize(t);
  if (dst.bytes() < bytes) fail(GR_EINVAL, "value buffer too small");
  if (t == DType::F64) {
    GR_CUDA(cudaMemcpyAsync(dst.get(), v.data(), bytes, cudaMemcpyHostToDevice, s));
  } else {
    std::vector<float> f(v.size());
    parallelChunks(static_cast<i64>(v.size()), [&](i64 b, i64 e) {
      for (i64 i = b; i < e; ++i) f[i] = static_cast<float>(v[i]);
    });
    GR_CUDA(cudaMemcpyAsync(dst.get(), f.data(), bytes, cudaMemcpyHostToDevice, s));
    GR_CUDA(cudaStreamSynchronize(s));  // f is released on return
  }
}
}  // namespace

void DeviceMatrix::updateValues(std::shared_ptr<HostMatrix> h) {
  const HostMatrix& H = *h;
  if (batch || !host || H.structureKey != host->structureKey || H.n != n || H.m != m || H.P != P ||
      H.valueType != vt || !H.sumRank.empty() || !host->sumRank.empty())
    fail(GR_EINVAL, "updateValues needs a CRS matrix with this matrix's structure");
  updateValues(H.offDiag, H.diag);
  host = std::move(h);
}

void DeviceMatrix::updateGlobalValues(const void* gVal, const void* gDiag, DType t) {
  if (t != DType::F64 && t != vt) fail(GR_EINVAL, "global values must be float64 or the coefficient type");
  if (batch || !host || !host->sumRank.empty() || host->format != GR_FORMAT_CRS ||
      static_cast<i64>(host->localSrc.size()) != m)
    fail(GR_EINVAL, "global values need a CRS matrix with its tile-local entry map");
  if (!gVal || !gDiag) fail(GR_EINVAL, "values must not be NULL");
  const HostMatrix& H = *host;
  ensureLocalCrs();
  if (!globalSrcOff.get()) {
    // Slot and entry maps into the global CRS order, built once.
    std::vector<i32> slotSrc(sell.slots, -1);
    const SellHost S = buildSell(H, 0);
    if (S.slots != sell.slots) fail(GR_EINVAL, "SELL layout mismatch");
    // The tile-local CRS entry behind every slot: the constructor's slot
    // assignment replayed.
    parallelChunks(n, [&](i64 b, i64 e) {
      for (i64 r = b; r < e; ++r) {
        const i64 c = r / 32, lane = r % 32;
        for (i64 k = 0; k < H.rowPtr[r + 1] - H.rowPtr[r]; ++k) {
          const i64 p = H.rowPtr[r] + k;
          slotSrc[S.base[c] + 32 * k + lane] = H.localSrc[p];
        }
      }
    });
    globalSrcOff.upload(H.localSrc);
    globalSrcSell.upload(slotSrc);
  }
  const size_t es = dtypeSize(t);
  DBuf gv(static_cast<size_t>(m) * es), gd(static_cast<size_t>(n) * es);
  GR_CUDA(cudaMemcpyAsync(gv.get(), gVal, static_cast<size_t>(m) * es, cudaMemcpyHostToDevice, stream));
  GR_CUDA(cudaMemcpyAsync(gd.get(), gDiag, static_cast<size_t>(n) * es, cudaMemcpyHostToDevice, stream));
  const i64 work = std::max<i64>(std::max<i64>(m, sell.slots), n);
  const int blocks = static_cast<int>(std::max<i64>(1, std::min<i64>(numSMs * 8, (work + 255) / 256)));
  int2* ent = vt == DType::F32 && !sell.compact ? sell.ent.as<int2>() : nullptr;
  const int* so = globalSrcOff.as<int>();
  const int* ss = globalSrcSell.as<int>();
  if (vt == DType::F32 && t == DType::F32)
    dev::globalValuesKernel<float, float><<<blocks, 256, 0, stream>>>(
        gv.as<float>(), gd.as<float>(), so, ss, iperm.as<int>(), offDiag.as<float>(), ent,
        ent ? nullptr : sell.val.as<float>(), diag.as<float>(), m, sell.slots, n);
  else if (vt == DType::F32)
    dev::globalValuesKernel<float, double><<<blocks, 256, 0, stream>>>(
        gv.as<double>(), gd.as<double>(), so, ss, iperm.as<int>(), offDiag.as<float>(), ent,
        ent ? nullptr : sell.val.as<float>(), diag.as<float>(), m, sell.slots, n);
  else
    dev::globalValuesKernel<double, double><<<blocks, 256, 0, stream>>>(
        gv.as<double>(), gd.as<double>(), so, ss, iperm.as<int>(), offDiag.as<double>(), nullptr,
        sell.val.as<double>(), diag.as<double>(), m, sell.slots, n);
  checkLaunch("global_values");
  GR_CUDA(cudaStreamSynchronize(stream));  // gv, gd are released on return
}

void DeviceMatrix::updateValues(const std::vector<double>& localOff, const std::vector<double>& tileDiag) {
  if (batch || !host || !host->sumRank.empty() || static_cast<i64>(localOff.size()) != m ||
      static_cast<i64>(tileDiag.size()) != n)
    fail(GR_EINVAL, "updateValues needs a CRS matrix's tile-local values and diagonal");
  const HostMatrix& H = *host;
  ensureLocalCrs();
  if (!sellSrc.get()) {
    // The constructor's slot assignment, recording entries instead of values.
    std::vector<i32> base(sell.nChunks + 1, 0);
    i64 acc = 0;
    for (i64 c = 0; c < sell.nChunks; ++c) {
      base[c] = static_cast<i32>(acc);
      i64 mx = 0;
      for (i64 r = c * 32; r < std::min<i64>(n, c * 32 + 32); ++r) mx = std::max(mx, H.rowPtr[r + 1] - H.rowPtr[r]);
      acc += 32 * mx;
    }
    if (acc != sell.slots) fail(GR_EINVAL, "SELL layout mismatch");
    std::vector<i32> src(sell.slots, -1);
    parallelChunks(n, [&](i64 b, i64 e) {
      for (i64 r = b; r < e; ++r)
        for (i64 k = 0; k < H.rowPtr[r + 1] - H.rowPtr[r]; ++k)
          src[base[r / 32] + 32 * k + r % 32] = static_cast<i32>(H.rowPtr[r] + k);
    });
    sellSrc.upload(src);
  }
  copyValuesInto(offDiag, localOff, vt, stream);
  copyValuesInto(diag, tileDiag, vt, stream);
  const int blocks = static_cast<int>(std::min<i64>(numSMs * 8, (sell.slots + 255) / 256 + 1));
  if (vt == DType::F32)
    dev::sellScatterKernel<float><<<blocks, 256, 0, stream>>>(
        sellSrc.as<int>(), offDiag.as<float>(), sell.compact ? nullptr : sell.ent.as<int2>(),
        sell.compact ? sell.val.as<float>() : nullptr, sell.slots);
  else
    dev::sellScatterKernel<double><<<blocks, 256, 0, stream>>>(sellSrc.as<int>(), offDiag.as<double>(), nullptr,
                                                               sell.val.as<double>(), sell.slots);
  checkLaunch("sell_scatter");
  GR_CUDA(cudaStreamSynchronize(stream));
}

// ---------------------------------------------------------------------------
namespace dev {

// y = A x. Every launch geometry (block size, grid, batch depth B) computes
// each row with the same sequential sum, so the autotuner's choice never
// changes y.
template <class MV, class VT, int B, bool C16>
__global__ void __launch_bounds__(512) spmvKernel(SellView<MV> A, const VT* __restrict__ x,
                                                   VT* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < A.nChunks; c += nWarps) {
    const int row = c * 32 + lane;
    const VT v = sellRowSum<VT, MV, VT, C16, B>(A, x, c, lane, row < A.n);
    if (row < A.n) y[row] = v;
  }
}

// Residual with an IEEE intermediate type I (float or double):
// r = (b - (d x + sum a x)) computed in I, stored as RT.
// Batches (seg): each system's rows with the block count a solve of it
// alone uses, its norm reduced over its own blocks into normOut[system].
template <class MV, class XT, class BT, class RT, class I, bool C16>
__global__ void __launch_bounds__(256) residualKernel(SellView<MV> A, const XT* __restrict__ x,
                                                       const BT* __restrict__ b,
                                                       RT* __restrict__ r, int normKind,
                                                       double* __restrict__ normOut,
                                                       double* partials, unsigned* counter, SegView seg) {
  __shared__ double smem[32];
  const SegPos sp = segPos(seg, A.n);
  const int lane = threadIdx.x & 31;
  const int nWarps = (sp.nb * blockDim.x) >> 5;
  const int cEnd = (sp.r1 + 31) >> 5;
  double part = redIdentity(normOp(normKind));
  for (int c = (sp.r0 >> 5) + ((sp.rank * blockDim.x + threadIdx.x) >> 5); c < cEnd; c += nWarps) {
    const int row = c * 32 + lane;
    const I sum = sellRowSum<I, MV, XT, C16>(A, x, c, lane, row < sp.r1);
    if (row < sp.r1) {
      RT res = cvt<RT>(sub(cvt<I>(__ldg(b + row)), sum));
      r[row] = res;
      if (normKind >= 0) part = normStep(part, toDouble(res), normKind);
    }
  }
  if (normKind < 0) return;
  double v[1] = {part};
  const int ops[1] = {normOp(normKind)};
  double out[1];
  blockReduce<1>(v, ops, smem);
  if (gridReduceRank<1>(v, ops, partials + sp.b0, counter + sp.sys, smem, out, sp.rank, sp.nb) &&
      threadIdx.x == 0)
    normOut[sp.sys] = normFinish(out[0], normKind);
}

// Residual with a double-word intermediate: x is double-word (two floats
// per entry) or float, the matrix float, b and r float.
template <bool XDW, bool C16>
__global__ void __launch_bounds__(256) residualDwKernel(SellView<float> A, const float* __restrict__ x,
                                                         const float* __restrict__ b,
                                                         float* __restrict__ r, int normKind,
                                                         double* __restrict__ normOut,
                                                         double* partials, unsigned* counter, SegView seg) {
  __shared__ double smem[32];
  const SegPos sp = segPos(seg, A.n);
  const int lane = threadIdx.x & 31;
  const int nWarps = (sp.nb * blockDim.x) >> 5;
  const int cEnd = (sp.r1 + 31) >> 5;
  double part = redIdentity(normOp(normKind));
  auto ld = [&](int i) -> dw {
    if (XDW) {
      float2 v = __ldg(reinterpret_cast<const float2*>(x) + i);
      return {v.x, v.y};
    }
    return {__ldg(x + i), 0.0f};
  };
  for (int c = (sp.r0 >> 5) + ((sp.rank * blockDim.x + threadIdx.x) >> 5); c < cEnd; c += nWarps) {
    const int row = c * 32 + lane;
    const bool live = row < sp.r1;
    dw sum = live ? dwTimesFp(ld(row), __ldg(A.diag + row)) : dw{0.0f, 0.0f};
    ChunkWalk<float, C16> w(A, c, lane);
    for (int k = 0; k < w.K; k += 4) {
      int cl[4];
      float a[4];
      w.template load<4>(A, k, cl, a);
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (cl[j] >= 0) sum = dwPlusDw(sum, dwTimesFp(ld(cl[j]), a[j]));
    }
    if (live) {
      dw res = dwPlusDw(dw{__ldg(b + row), 0.0f}, dwNeg(sum));
      float rv = dwToFloat(res);
      r[row] = rv;
      if (normKind >= 0) part = normStep(part, static_cast<double>(rv), normKind);
    }
  }
  if (normKind < 0) return;
  double v[1] = {part};
  const int ops[1] = {normOp(normKind)};
  double out[1];
  blockReduce<1>(v, ops, smem);
  if (gridReduceRank<1>(v, ops, partials + sp.b0, counter + sp.sys, smem, out, sp.rank, sp.nb) &&
      threadIdx.x == 0)
    normOut[sp.sys] = normFinish(out[0], normKind);
}

template <class T>
__global__ void __launch_bounds__(256) normKernel(const T* __restrict__ x, int n, int kind,
                                                   double* __restrict__ out, double* partials,
                                                   unsigned* counter) {
  __shared__ double smem[32];
  double part = redIdentity(normOp(kind));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    part = normStep(part, toDouble(__ldg(x + i)), kind);
  double v[1] = {part};
  const int ops[1] = {normOp(kind)};
  double res[1];
  blockReduce<1>(v, ops, smem);
  if (gridReduce<1>(v, ops, partials, counter, smem, res) && threadIdx.x == 0)
    *out = normFinish(res[0], kind);
}

template <class T>
__global__ void permuteKernel(const T* __restrict__ src, T* __restrict__ dst,
                              const int* __restrict__ iperm, int n, bool toTile) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    int g = __ldg(iperm + p);
    if (toTile) dst[p] = src[g];
    else dst[g] = src[p];
  }
}

}  // namespace dev

// ---------------------------------------------------------------------------
namespace {

}  // namespace

namespace {
template <class MV, class VT>
void spmvT(DeviceMatrix& A, const void* x, void* y, const SpmvTuning& g, cudaStream_t s) {
  // chunksPerWarp 0: the untuned geometry (A.spmvBlocks(), at most 8 blocks
  // per SM, warps striding over the chunks).
  const int warps = g.block / 32;
  const int blocks = g.chunksPerWarp == 0
                         ? A.spmvBlocks()
                         : std::max(1, std::min((A.sell.nChunks + warps * g.chunksPerWarp - 1) /
                                                    (warps * g.chunksPerWarp),
                                                A.numSMs * 64));
  const auto* xv = static_cast<const VT*>(x);
  auto* yv = static_cast<VT*>(y);
  const bool c16 = A.sell.compact;
  auto kernel = g.batch == 4    ? (c16 ? dev::spmvKernel<MV, VT, 4, true> : dev::spmvKernel<MV, VT, 4, false>)
                : g.batch == 16 ? (c16 ? dev::spmvKernel<MV, VT, 16, true> : dev::spmvKernel<MV, VT, 16, false>)
                                : (c16 ? dev::spmvKernel<MV, VT, 8, true> : dev::spmvKernel<MV, VT, 8, false>);
  kernel<<<blocks, g.block, 0, s>>>(sellView<MV>(A), xv, yv);
}

SpmvTuning& tuningFor(DeviceMatrix& A, DType t) { return A.spmvTuning[t == DType::F64 ? 1 : 0]; }
}  // namespace

void launchSpmv(DeviceMatrix& A, const void* x, void* y, DType t, cudaStream_t s) {
  const SpmvTuning& g = tuningFor(A, t);
  if (A.vt == DType::F32 && t == DType::F32) {
    spmvT<float, float>(A, x, y, g, s);
  } else if (A.vt == DType::F32 && t == DType::F64) {
    spmvT<float, double>(A, x, y, g, s);
  } else if (A.vt == DType::F64 && t == DType::F64) {
    spmvT<double, double>(A, x, y, g, s);
  } else {
    fail(GR_EUNSUPPORTED, std::string("spmv with ") + dtypeName(A.vt) + " coefficients and " +
                              dtypeName(t) + " vectors");
  }
  checkLaunch("spmv");
}

SpmvTuning tuneSpmv(DeviceMatrix& A, DType t, int reps) {
  if (t != DType::F32 && t != DType::F64) fail(GR_EINVAL, "spmv tuning needs float32 or float64 vectors");
  if (A.vt == DType::F64 && t == DType::F32) fail(GR_EUNSUPPORTED, "spmv with float64 coefficients and float32 vectors");
  if (reps < 1 || reps > 1000) fail(GR_EINVAL, "reps must be 1..1000");
  const size_t bytes = static_cast<size_t>(A.n) * dtypeSize(t);
  DBuf x(bytes), y(bytes);
  GR_CUDA(cudaMemsetAsync(x.get(), 0, bytes, A.stream));
  // Every timed launch starts with L2 flushed (a 256 MB write, twice the
  // B200's 126 MB L2), as a solve meets a matrix larger than L2: a warm L2
  // would favour geometries that a solve never sees.
  const size_t flushBytes = size_t(256) << 20;
  DBuf flush(flushBytes);
  cudaEvent_t e0, e1;
  GR_CUDA(cudaEventCreate(&e0));
  GR_CUDA(cudaEventCreate(&e1));
  SpmvTuning& slot = tuningFor(A, t);
  const SpmvTuning keep = slot;
  SpmvTuning best = keep;
  float bestMs = 1e30f;
  try {
    for (int block : {128, 256, 512})
      for (int cpw : {0, 1, 2, 4, 8})
        for (int batch : {4, 8, 16}) {
          if (cpw == 0 && block != 256) continue;  // the untuned geometry
          slot = SpmvTuning{block, cpw, batch, false, 0.0f};
          launchSpmv(A, x.get(), y.get(), t, A.stream);  // warm-up
          float ms = 0;
          for (int r = 0; r < reps; ++r) {
            GR_CUDA(cudaMemsetAsync(flush.get(), r & 0xFF, flushBytes, A.stream));
            GR_CUDA(cudaEventRecord(e0, A.stream));
            launchSpmv(A, x.get(), y.get(), t, A.stream);
            GR_CUDA(cudaEventRecord(e1, A.stream));
            GR_CUDA(cudaEventSynchronize(e1));
            float one = 0;
            GR_CUDA(cudaEventElapsedTime(&one, e0, e1));
            ms += one;
          }
          if (ms < bestMs) {
            bestMs = ms;
            best = slot;
          }
        }
  } catch (...) {
    slot = keep;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  best.tuned = true;
  best.ms = bestMs / static_cast<float>(reps);
  slot = best;
  GR_CUDA(cudaStreamSynchronize(A.stream));
  return best;
}

float timeSpmv(DeviceMatrix& A, const void* x, void* y, DType t, int reps, bool flushL2) {
  if (reps < 1 || reps > 10000) fail(GR_EINVAL, "reps must be 1..10000");
  // Each launch is timed alone between two events on the matrix's stream;
  // with flushL2, a 256 MB write (twice the B200's 126 MB L2) precedes it.
  const size_t flushBytes = flushL2 ? size_t(256) << 20 : 0;
  DBuf flush(flushBytes > 0 ? flushBytes : 16);
  cudaEvent_t e0, e1;
  GR_CUDA(cudaEventCreate(&e0));
  GR_CUDA(cudaEventCreate(&e1));
  float total = 0;
  try {
    launchSpmv(A, x, y, t, A.stream);  // warm-up
    for (int r = 0; r < reps; ++r) {
      if (flushL2) GR_CUDA(cudaMemsetAsync(flush.get(), r & 0xFF, flushBytes, A.stream));
      GR_CUDA(cudaEventRecord(e0, A.stream));
      launchSpmv(A, x, y, t, A.stream);
      GR_CUDA(cudaEventRecord(e1, A.stream));
      GR_CUDA(cudaEventSynchronize(e1));
      float one = 0;
      GR_CUDA(cudaEventElapsedTime(&one, e0, e1));
      total += one;
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return total / static_cast<float>(reps);
}

void launchResidual(DeviceMatrix& A, const void* x, DType xt, const void* b, DType bt, void* r,
                    DType rt, DType inter, int normKind, double* normOut, cudaStream_t s) {
  int blocks = A.spmvBlocks();
  double* part = A.partials.as<double>();
  unsigned* cnt = A.counter.as<unsigned>();
  dev::SegView seg;
  if (A.batch) {
    // Every system over its own rows and blocks (the row-chunk tables of
    // the batch), its norm into normOut[system].
    const BatchSeg& B = *A.batch;
    blocks = B.chunkGrid;
    seg.blockSys = B.chunkSys.as<int>();
    seg.blockRank = B.chunkRank.as<int>();
    seg.sysBlocks = B.chunkBlocks.as<int>();
    seg.sysBlock0 = B.chunkBlock0.as<int>();
    seg.sysRow0 = B.row0.as<int>();
    seg.sysRowEnd = B.rowEnd.as<int>();
    part = B.partials.as<double>();
    cnt = B.counters.as<unsigned>();
  }
  auto bad = [&]() {
    fail(GR_EUNSUPPORTED, std::string("residual with x=") + dtypeName(xt) + " b=" + dtypeName(bt) +
                              " r=" + dtypeName(rt) + " intermediate=" + dtypeName(inter) +
                              " coefficients=" + dtypeName(A.vt));
  };
  if (inter == DType::DW) {
    if (A.vt != DType::F32 || bt != DType::F32 || rt != DType::F32) bad();
    if (xt != DType::DW && xt != DType::F32) bad();
    const bool c16 = A.sell.compact;
    auto kernel = xt == DType::DW ? (c16 ? dev::residualDwKernel<true, true> : dev::residualDwKernel<true, false>)
                                  : (c16 ? dev::residualDwKernel<false, true> : dev::residualDwKernel<false, false>);
    kernel<<<blocks, 256, 0, s>>>(sellView<float>(A), static_cast<const float*>(x), static_cast<const float*>(b),
                                  static_cast<float*>(r), normKind, normOut, part, cnt, seg);
    checkLaunch("residual_dw");
    return;
  }
  if (xt == DType::DW) bad();
#define GR_RES(MV, XT, BT, RT, IT)                                                                        \
  (A.sell.compact ? dev::residualKernel<MV, XT, BT, RT, IT, true> : dev::residualKernel<MV, XT, BT, RT, IT, false>) \
      <<<blocks, 256, 0, s>>>(sellView<MV>(A), static_cast<const XT*>(x), static_cast<const BT*>(b),        \
                              static_cast<RT*>(r), normKind, normOut, part, cnt, seg)
  const bool mf = A.vt == DType::F32;
  const int key = (xt == DType::F64) * 8 + (bt == DType::F64) * 4 + (rt == DType::F64) * 2 +
                  (inter == DType::F64);
  if (mf) {
    switch (key) {
      case 0: GR_RES(float, float, float, float, float); break;
      case 1: GR_RES(float, float, float, float, double); break;
      case 3: GR_RES(float, float, float, double, double); break;  // a float64 working type over float32 x and b
      case 7: GR_RES(float, float, double, double, double); break;
      case 9: GR_RES(float, double, float, float, double); break;
      case 11: GR_RES(float, double, float, double, double); break;
      case 15: GR_RES(float, double, double, double, double); break;
      default: bad();
    }
  } else {
    switch (key) {
      case 9: GR_RES(double, double, float, float, double); break;
      case 11: GR_RES(double, double, float, double, double); break;
      case 15: GR_RES(double, double, double, double, double); break;
      default: bad();
    }
  }
#undef GR_RES
  checkLaunch("residual");
}

void launchNormN(DeviceMatrix& A, const void* x, i64 n, DType t, int normKind, double* out, cudaStream_t s) {
  const int blocks = static_cast<int>(std::max<i64>(1, std::min<i64>(A.redBlocks, (n + 255) / 256)));
  if (t == DType::F32)
    dev::normKernel<float><<<blocks, 256, 0, s>>>(static_cast<const float*>(x), static_cast<int>(n), normKind, out,
                                                  A.partials.as<double>(), A.counter.as<unsigned>());
  else if (t == DType::F64)
    dev::normKernel<double><<<blocks, 256, 0, s>>>(static_cast<const double*>(x), static_cast<int>(n), normKind,
                                                   out, A.partials.as<double>(), A.counter.as<unsigned>());
  else
    fail(GR_EUNSUPPORTED, "norm of a twofloat32 vector");
  checkLaunch("norm");
}

void launchNorm(DeviceMatrix& A, const void* x, DType t, int normKind, double* out, cudaStream_t s) {
  launchNormN(A, x, A.n, t, normKind, out, s);
}

void launchPermute(DeviceMatrix& A, const void* src, void* dst, DType t, bool toTile, cudaStream_t s) {
  const int blocks = std::max(1, std::min(A.redBlocks, (A.n + 255) / 256));
  if (dtypeSize(t) == 4)
    dev::permuteKernel<float><<<blocks, 256, 0, s>>>(static_cast<const float*>(src), static_cast<float*>(dst),
                                                     A.iperm.as<int>(), A.n, toTile);
  else
    dev::permuteKernel<double><<<blocks, 256, 0, s>>>(static_cast<const double*>(src), static_cast<double*>(dst),
                                                      A.iperm.as<int>(), A.n, toTile);
  checkLaunch("permute");
}

}  // namespace gr

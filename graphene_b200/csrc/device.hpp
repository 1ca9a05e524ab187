// Device-side data structures of graphene_b200 and the host wrappers that
// launch its CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "common.hpp"
#include "host_matrix.hpp"

namespace gr {

void cudaCheck(cudaError_t e, const char* what);
#define GR_CUDA(call) ::gr::cudaCheck((call), #call)

// Counts every kernel launch made through this library. Launches recorded
// while a CUDA graph is being captured are not counted; graph replays add
// the graph's kernel count instead.
void noteLaunch(int count = 1);
i64 launchCount();
void setCapturing(bool on);
bool capturing();
// Kernels recorded while capturing (per thread).
i64 capturedCount();

// Owning device allocation.
class DBuf {
 public:
  DBuf() = default;
  explicit DBuf(size_t bytes) { alloc(bytes); }
  ~DBuf() { release(); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p_(o.p_), bytes_(o.bytes_), dev_(o.dev_) { o.p_ = nullptr; o.bytes_ = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p_ = o.p_; bytes_ = o.bytes_; dev_ = o.dev_; o.p_ = nullptr; o.bytes_ = 0; }
    return *this;
  }
  void alloc(size_t bytes);
  void release();
  void* get() const { return p_; }
  template <class T> T* as() const { return static_cast<T*>(p_); }
  size_t bytes() const { return bytes_; }
  template <class T>
  void upload(const std::vector<T>& v) {
    alloc(std::max<size_t>(1, v.size()) * sizeof(T));
    if (!v.empty()) GR_CUDA(cudaMemcpy(p_, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  }

 private:
  void* p_ = nullptr;
  size_t bytes_ = 0;
  int dev_ = 0;
};

// Values converted to the stored coefficient type (float or double).
void uploadValues(DBuf& dst, const std::vector<double>& v, DType t);

// Sliced-ELLPACK (chunk height 32) copy of the off-diagonal part in tile
// order. Row r of chunk c keeps its entries in the reference's tile-local
// column order at slots base[c] + 32*k + (r % 32); padding slots hold
// column -1 and value 0. Used by SpMV and residual kernels.
//
// Two column encodings. The 32-bit layout stores each slot's tile-order
// column. The 16-bit layout stores column - row as a 16-bit integer (0:
// padding) and moves the columns too far from their row (|column - row| >
// 32767, code -32768) to a side list in slot order, with the count of such
// entries before each chunk: for a float matrix 6 bytes a slot instead of
// 8. Both give every row the same terms in the same order.
struct SellMatrix {
  i32 n = 0, nChunks = 0;
  i64 slots = 0;
  bool compact = false;  // the 16-bit layout
  i64 far = 0;           // entries in the far list
  DBuf base;     // i32[nChunks + 1]
  DBuf ent;      // 32-bit layout, float coefficients: int2 {tile-order column, value bits} [slots]
  DBuf col;      // 32-bit layout, double coefficients: i32 tile-order column [slots]
  DBuf val;      // values [slots]: double coefficients, or the 16-bit layout
  DBuf d16;      // 16-bit layout: i16 column - row [slots]
  DBuf farCol;   // 16-bit layout: i32 far columns [far]
  DBuf farBase;  // 16-bit layout: i32[nChunks + 1], far entries before each chunk
};

// Host image of the SELL layout of H (both encodings' arrays; the 16-bit
// ones filled when `compact`). layout: 0 or -1 (automatic) the 32-bit
// layout, 1 the 16-bit layout (GR_EUNSUPPORTED when a chunk has more than
// 64 far entries).
struct SellHost {
  i64 slots = 0;
  bool compact = false;
  std::vector<i32> base, col;  // col: tile-order column of every slot (-1 padding)
  std::vector<double> val;
  std::vector<int16_t> d16;
  std::vector<i32> farCol, farBase;
  i64 maxChunkFar = 0;  // most far entries in one chunk (the 16-bit layout allows 64)
};
SellHost buildSell(const HostMatrix& H, int layout);
// Decodes the 16-bit arrays of S chunk by chunk, in the order the device's
// warps walk them, and checks every slot against the 32-bit columns;
// throws on the first mismatch.
void checkSellDecode(const SellHost& S, i64 n);

// Level schedule of one sweep over all tiles: for each tile its levels, for
// each level its rows, and for each row its entries stored level-major
// (slot = levelSlotStart + k * levelRows + q), so a level's rows load their
// k-th entries with one coalesced access.
struct LevelSchedule {
  i32 numLevels = 0;
  i32 maxLevelRows = 0;
  i64 slots = 0;
  DBuf tileLvlStart;  // i32[P + 1]
  DBuf lvlRowStart;   // i32[L + 1]
  DBuf lvlSlotStart;  // i64[L + 1]
  DBuf rows;          // i32 tile-order row per level row
  DBuf col;           // i32 tile-order column per slot, -1 = padding
  DBuf src;           // i32 index into the local CRS values per slot, -1 = padding
};

// Byte stream of a tile's whole ILU application, consumed in order by the
// streamed substitution kernel. Per tile:
//   tile header  int4 {numLowerLevels, numUpperLevels, 0, 0}
//   per level    int4 {k rows, E entries per row, hasInv, 0}
//                rows  k x int32 tile-local row ids            (16-byte padded)
//                inv   k x value type inverse diagonal (if hasInv)    (padded)
//                cols  E*k x int32 tile-local columns, -1 pad, entry-major
//                vals  E*k x value type, entry-major                  (padded)
// lower levels (forward substitution, ascending columns) first, then upper
// levels (backward substitution, descending columns). The template holds the
// structure; a solver copies it and packs its factor values and inverse
// diagonal in (valPos / valSrc, invPos / invSrc, element indices in units of
// the value type).
struct SweepStream {
  bool dilu = false;
  i64 bytes = 0;
  i64 maxLevelBytes = 0;
  i64 maxSpanBytes = 0;  // largest span of two consecutive levels (ring sizing)
  i64 nVal = 0, nInv = 0;
  DBuf tileOffset;  // i64[P + 1]
  DBuf templ;       // bytes
  DBuf valPos, valSrc, invPos, invSrc;  // i32
  // Level table: per level int4 {byte offset of its header in the tile's
  // stream, k, E, hasInv}; tile T's levels are [tileLevel[T], tileLevel[T+1]).
  DBuf levelTable;  // int4
  DBuf tileLevel;   // i32[P + 1]
  i64 numLevels = 0;
  i32 maxTileLevels = 0;
  i32 maxLevelRows = 0;
  i32 maxEntries = 0;
};

// Host copy of a SweepStream (built on the host, then uploaded).
struct HostStream {
  std::vector<uint8_t> bytes;
  std::vector<i64> tileOffset;
  std::vector<i32> valPos, valSrc, invPos, invSrc;
  i64 maxLevelBytes = 0;
  // Largest distance from the start of a level (the tile header for the
  // first) to the end of the next level: the streamed kernel keeps two
  // consecutive levels in its ring.
  i64 maxSpanBytes = 0;
  std::vector<int4> levelTable;  // see SweepStream::levelTable
  std::vector<i32> tileLevel;
  i32 maxTileLevels = 0, maxLevelRows = 0, maxEntries = 0;
};
// Chunks of the streamed kernel's shared-memory ring.
constexpr int kRingChunksHost = 8;
HostStream buildIluStream(const HostMatrix& H, bool dilu, DType vt);
// log2 of the ring size the streamed kernel uses for a given largest
// two-level span.
int ringLog2ForLevel(i64 maxSpanBytes);
// Replays the streamed kernel's reads on the host; throws GR_EINVAL on any
// out-of-range index, ordering or ring-capacity violation.
void checkIluStream(const HostMatrix& H, const HostStream& S, bool dilu, DType vt, int ringLog2);

// Level blocks for the host-scheduled ring kernel (kernels_ring.cu). Per
// tile, the levels in execution order (lower ascending, then upper
// descending). A level block (every segment 16-byte padded) is, in the
// compact layout (blocks of at most 65535 rows):
//   rows  k x u16 block-local row ids
//   inv   k x value type inverse diagonal (upper levels, DILU)
//   cols  E*k x u16 columns, entry-major
//   vals  E*k x value type, entry-major
// and otherwise (the wide layout):
//   rows  k x i32
//   inv   k x value type (upper levels, DILU)
//   ents  E*k entries, entry-major, {i32 column, value}: 8 bytes for float,
//         16 for double ({column, 0, value})
// Padding entries use column nRows (a zero slot of the kernel's x slice) and
// value 0. One int4 per level (RingLevelCode): k; E, the entries' offset
// and the sweep; the ring offset and the block's size; issueAfter. The
// kernel copies a level's block into its shared-memory ring at `ring offset`
// once the tile's level `issueAfter` has been consumed (-1: at the start);
// the host chose the offsets so that a copy never overwrites a level still
// to be consumed, and so that every level is copied at least one level
// before it is needed.
constexpr int kRingBarriers = 16;
constexpr int kRingUpperBit = 1 << 30;
// Field packing of a level's int4: y = E | (entries offset / 16) << 14 |
// upper << 30 | record << 31, z = ring offset | (block bytes / 16) << 18.
constexpr int kRingEBits = 14, kRingOffBits = 18;
constexpr uint32_t kRingRecordBit = 1u << 31;
struct RingLevelCode {
  __host__ __device__ static int k(const int4 m) { return m.x; }
  __host__ __device__ static int E(const int4 m) { return m.y & ((1 << kRingEBits) - 1); }
  __host__ __device__ static uint32_t ents(const int4 m) {
    return ((static_cast<uint32_t>(m.y) >> kRingEBits) & 0xFFFFu) << 4;
  }
  __host__ __device__ static bool upper(const int4 m) { return (m.y & kRingUpperBit) != 0; }
  __host__ __device__ static bool record(const int4 m) { return (static_cast<uint32_t>(m.y) & kRingRecordBit) != 0; }
  __host__ __device__ static uint32_t ringOffset(const int4 m) {
    return static_cast<uint32_t>(m.z) & ((1u << kRingOffBits) - 1);
  }
  __host__ __device__ static uint32_t bytes(const int4 m) { return (static_cast<uint32_t>(m.z) >> kRingOffBits) << 4; }
  __host__ __device__ static int issueAfter(const int4 m) { return m.w; }
};
constexpr long long kRingCompactRows = 65535;  // largest block (rows + zero slot) of the compact layout

// Byte offsets of a level block's inverse diagonal, entries (columns, or
// column/value pairs) and values, and its size.
//
// Record levels (compact layout, float values, exactly 3 entries a row, as
// a 7-point stencil's lower or upper part has): a row is one 16-byte record
// {v0, v1, v2, c0 | c1 << 16} at 16 q, then, after all of them, a 4-byte
// word {c2 | row << 16} at ents + 4 q, or with an inverse diagonal an 8-byte
// pair {c2 | row << 16, inv} at ents + 8 q. Two shared-memory loads a row
// instead of seven, at the bytes of the column-major compact layout.
__host__ __device__ inline bool ringRecordLevel(uint32_t E, uint32_t valueBytes, bool compact) {
  return compact && valueBytes == 4 && E == 3;
}
struct RingLevelLayout {
  uint32_t inv, ents, vals, bytes;
};
__host__ __device__ inline RingLevelLayout ringLevelLayout(uint32_t k, uint32_t E, bool hasInv, uint32_t valueBytes,
                                                           bool compact, bool record = false) {
  if (record) {
    const uint32_t recB = ((hasInv ? 8u : 4u) * k + 15u) & ~15u;
    return RingLevelLayout{16u * k, 16u * k, 0u, 16u * k + recB};
  }
  const uint32_t idB = compact ? 2u : 4u;
  const uint32_t rowsB = (idB * k + 15u) & ~15u;
  const uint32_t invB = hasInv ? ((valueBytes * k + 15u) & ~15u) : 0u;
  if (compact) {
    const uint32_t colsB = (2u * E * k + 15u) & ~15u;
    const uint32_t valsB = (valueBytes * E * k + 15u) & ~15u;
    return RingLevelLayout{rowsB, rowsB + invB, rowsB + invB + colsB, rowsB + invB + colsB + valsB};
  }
  const uint32_t entBytes = valueBytes == 4 ? 8u : 16u;
  const uint32_t entB = (entBytes * E * k + 15u) & ~15u;
  return RingLevelLayout{rowsB, rowsB + invB, rowsB + invB, rowsB + invB + entB};
}

// What the default ring size is chosen for: the SM count, shared memory per
// SM, the shared memory the runtime reserves per block, and the blocks per SM
// that threads and registers allow. The default ring is the size (between the
// smallest that places and max(16 KB, 4 x the largest level)) that needs the
// fewest waves of blocks, the largest such.
struct RingBudget {
  i32 numSMs = 148;
  i64 smemPerSM = 233472;
  i64 reservedPerBlock = 1024;
  i32 maxBlocksPerSM = 16;  // the ring kernel's thread and register limit on B200
};
// What a level ring holds: the ILU(0) / DILU forward and backward
// substitution (each row's lower, then upper entries, halo dropped), or one
// Gauss-Seidel sweep over the lower levels with each row's entries in
// tile-local order (all of them; or, for a sweep that starts from x = 0,
// only the lower ones, the others multiplying zero).
//
// Gauss-Seidel rings address x through one shared-memory array per tile of
// 2 nRows + nHalo + 1 slots: [0, nRows) the values of this sweep, [nRows,
// 2 nRows) the tile's values at the start of the sweep, then the halo
// values at the start of the sweep (the reference's halo exchange,
// gauss-seidel/Solver.cpp:61) and a zero slot for padding entries. An entry
// with tile-local column c of row i reads slot c when c < i and nRows + c
// otherwise (halo columns are >= nRows). The row's diagonal takes the
// inverse diagonal's place in the level block, and the right-hand side
// (nRows more slots) follows the array. In place (gsInPlace: every upper
// entry of a tile lies in a later level than its row), the array is nRows +
// nHalo + 1 slots: the start values are loaded into [0, nRows) and
// overwritten row by row, and an entry reads slot c whatever its side.
enum class RingKind { Ilu = 0, GaussSeidel = 1, GaussSeidelLower = 2 };

struct HostRing {
  RingKind kind = RingKind::Ilu;
  i64 maxXSlots = 0;               // Gauss-Seidel: shared-memory x slots per tile (with the right-hand side)
  bool gsInPlace = false;          // Gauss-Seidel: no sweep-start copy (upper entries read their own slot)
  std::vector<i32> haloStart;      // Gauss-Seidel: P + 1 offsets into haloSrc
  std::vector<i32> haloSrc;        // Gauss-Seidel: tile-order index of every tile's halo cells
  std::vector<uint8_t> bytes;
  std::vector<i64> tileOffset;  // P + 1
  std::vector<int4> meta;       // 1 per level
  std::vector<i32> tileLevel;   // P + 1
  std::vector<i32> valPos, valSrc, invPos, invSrc;  // element positions (value type units)
  i64 ringBytes = 0, maxLevelBytes = 0, maxGroupRows = 0;
  i32 maxTileLevels = 0;
  i32 group = 1;                // tiles per thread block
  bool compact = false;         // 16-bit row and column ids
  std::vector<i32> groupStart;  // first tile-order row of every block, and n
};
// Shared memory of one ring-kernel block besides the ring: barriers, the
// level table and the block's slice of x (plus its zero slot).
// Header: kRingBarriers full and kRingBarriers empty mbarriers, one for the
// level table, padded to 16 bytes.
constexpr i64 kRingHeader = (8 * (2 * kRingBarriers + 1) + 15) / 16 * 16;
inline i64 ringFixedSmemSlots(i32 maxTileLevels, i64 xSlots, i64 vectorBytes) {
  return kRingHeader + 16 * static_cast<i64>(maxTileLevels) + xSlots * vectorBytes;
}
inline i64 ringFixedSmem(i32 maxTileLevels, i64 maxGroupRows, i64 vectorBytes) {
  return ringFixedSmemSlots(maxTileLevels, maxGroupRows + 1, vectorBytes);
}
// One thread block runs `group` consecutive tiles in lockstep (tileOffset,
// tileLevel and meta are then per block). ringBytes 0: the default (RingBudget).
// The compact layout is used when every block has at most kRingCompactRows
// rows and `allowCompact`.
// records: use record levels where they apply (ringRecordLevel).
HostRing buildLevelRing(const HostMatrix& H, bool dilu, DType vt, i64 ringBytes, i32 group,
                        const RingBudget& budget = RingBudget{}, bool allowCompact = true,
                        RingKind kind = RingKind::Ilu, bool records = false);
// Replays the kernel's copies and reads on the host; throws GR_EINVAL on an
// out-of-range index, a dependency-order violation, a copy that would
// overwrite a level not yet consumed, or a copy issued too late.
void checkLevelRing(const HostMatrix& H, const HostRing& R, bool dilu, DType vt);
struct LevelRing {
  RingKind kind = RingKind::Ilu;
  bool dilu = false;
  i64 bytes = 0, ringBytes = 0, nVal = 0, nInv = 0, maxGroupRows = 0, maxXSlots = 0;
  i32 maxTileLevels = 0, group = 1, numGroups = 0;
  bool compact = false;
  bool gsInPlace = false;
  DBuf tileOffset, templ, meta, tileLevel, groupStart, valPos, valSrc, invPos, invSrc;
  DBuf haloStart, haloSrc;  // Gauss-Seidel rings
};

// Kinds of entries a schedule keeps per row.
enum class SweepEntries {
  Lower,        // tile-local columns below the row, ascending (ILU forward)
  UpperDesc,    // tile-local columns above the row (non-halo), descending (ILU backward)
  All           // every off-diagonal entry in tile-local order (Gauss-Seidel)
};

// Launch geometry of the SpMV kernel: threads per block, SELL chunks per
// warp (grid size; 0 = the untuned grid), and entries whose loads are issued
// together (batch).
struct SpmvTuning {
  int block = 256, chunksPerWarp = 0, batch = 8;
  bool tuned = false;
  float ms = 0;  // mean time of the chosen geometry when tuned
};

// A batch of independent systems stored as one block-diagonal device matrix:
// system s owns tile-order rows [rowBegin[s], rowBegin[s] + rowReal[s]) (its
// own tile layout, unchanged) followed by padding rows up to the next
// multiple of 32, so that no SELL chunk mixes systems. Two block tables split
// the launches of the Krylov kernels per system: `chunk` for the row-chunk
// kernels (each system gets the block count a solve of it alone would use)
// and `elem` for the elementwise ones. tileSys maps a tile to its system.
struct BatchSeg {
  int systems = 0;
  std::vector<i64> rowBegin, rowReal;
  std::vector<i32> tileBegin;                 // first tile of each system, and P
  DBuf row0, rowEnd;                          // i32[systems]
  DBuf chunkSys, chunkRank, chunkBlocks, chunkBlock0;
  DBuf elemSys, elemRank, elemBlocks, elemBlock0;
  int chunkGrid = 0, elemGrid = 0;
  DBuf partials, counters;                    // per-block partials, per-system arrival counters
  DBuf tileSys;                               // i32[P]
};

struct DeviceMatrix {
  std::shared_ptr<HostMatrix> host;
  int device = 0;
  int numSMs = 148;
  cudaStream_t ownStream = nullptr;
  cudaStream_t stream = nullptr;
  i32 n = 0, P = 0;
  i64 m = 0;
  DType vt = DType::F32;

  SellMatrix sell;
  DBuf diag;       // value type [n]
  DBuf tileStart;  // i32[P + 1]
  DBuf iperm;      // i32[n]

  // Tile-local CRS in tile order (for the factorisation), built on demand.
  bool haveLocalCrs = false;
  DBuf rowPtr;     // i32[n + 1]
  DBuf colLocal;   // i32[m]
  DBuf offDiag;    // value type [m]

  // Schedules, built on demand.
  std::unique_ptr<LevelSchedule> lowerSched, upperSched, gsSched;
  std::unique_ptr<SweepStream> iluStream[2];  // [dilu]
  SweepStream& iluSweepStream(bool dilu);
  std::map<std::tuple<bool, i64, i32, bool, int, bool>, std::unique_ptr<LevelRing>>
      levelRings;  // [(dilu, ring bytes, group, compact allowed, kind, record levels)]
  LevelRing& levelRing(bool dilu, i64 ringBytes, i32 group, bool allowCompact = true,
                       RingKind kind = RingKind::Ilu, bool records = false);

  // Device error word written by kernels whose bounded waits ran out
  // (GR_ETIMEOUT); 0 when clean.
  DBuf errFlag;  // int

  // Reduction scratch: per-block partials and an arrival counter.
  DBuf partials;   // double[maxBlocks * 8]
  DBuf counter;    // unsigned[16]
  int redBlocks = 0;

  // Small device scratch for norms returned to the host.
  DBuf scalarOut;  // double[8]

  // Staging vectors of host-buffer solves (b, x and a permutation buffer),
  // kept across solvers of this matrix so that a solve from host memory
  // allocates nothing after the first. Solves of one matrix are ordered on
  // its stream, so they never use them at the same time.
  DBuf stage[3];
  void* staging(int i, size_t bytes) {
    if (stage[i].bytes() < bytes) stage[i].alloc(bytes);
    return stage[i].get();
  }

  explicit DeviceMatrix(std::shared_ptr<HostMatrix> h);
  ~DeviceMatrix();

  void ensureLocalCrs();
  // Replaces the coefficients by those of h, a matrix with this matrix's
  // structure (equal HostMatrix::structureKey, CRS): the new tile-local
  // values and diagonal are uploaded in place and scattered into the SpMV
  // layout on the device; every layout array, schedule and level-ring
  // template stays. Solver trees on this matrix then need refresh().
  void updateValues(std::shared_ptr<HostMatrix> h);
  // The same from values already in this matrix's layout: tile-local CRS
  // off-diagonals (m) and the tile-ordered diagonal (n), in FP64 (rounded
  // to the coefficient type here). The host matrix's own values go stale.
  void updateValues(const std::vector<double>& localOff, const std::vector<double>& tileDiag);
  DBuf sellSrc;  // tile-local CRS entry of every SELL slot (-1: padding), built on the first update
  // The same from global CRS values (natural order; host pointers to m and
  // n values of type t, FP64 or the coefficient type), gathered into place
  // on the device: no host-side permutation.
  void updateGlobalValues(const void* gVal, const void* gDiag, DType t);
  DBuf globalSrcOff, globalSrcSell;  // global CRS entry of every local entry / SELL slot (-1: padding)
  LevelSchedule& schedule(SweepEntries kind);
  // Grid of the row-chunk kernels (SpMV-dot, residual, PBiCGStab init): a
  // block per 8 chunks, at most one wave of resident blocks (sellGridCap).
  int spmvBlocks() const;
  int sellGridCap() const;
  mutable int sellCap = 0;
  SpmvTuning spmvTuning[2];  // [float32 vectors, float64 vectors]
  // Set for a batch of systems (makeBatch): the Krylov kernels then keep one
  // state per system.
  std::unique_ptr<BatchSeg> batch;
  void makeBatch(const std::vector<i64>& rowBegin, const std::vector<i64>& rowReal,
                 const std::vector<i32>& tileBegin);
};

// Raises the dynamic shared-memory limit of kernel `fn` on the current device
// to at least `bytes`. The limit is shared by every thread of the process,
// so it is only ever raised (a lower request never undoes a higher one that
// another thread's launch relies on).
void ensureDynamicSmem(const void* fn, size_t bytes);
// Runs the bounded-wait self-test (selftest.cu): the status the waiting
// kernel reported (GR_ETIMEOUT when the bound works) and how long it waited.
void selftestWaitTimeout(int32_t* status, int64_t* elapsedNs);
// Asks for the largest shared-memory carveout for `fn` (once per device), so
// that as many of its blocks as shared memory allows are resident per SM.
void preferSharedCarveout(const void* fn);

// ---- launchers -------------------------------------------------------

// y = A x (reference CRSMatrix::spmv). xt == yt.
void launchSpmv(DeviceMatrix& A, const void* x, void* y, DType t, cudaStream_t s);

// Blocks of 256 threads per SM that every row-chunk Krylov kernel
// (PBiCGStab init, both SpMV-dot kernels; float and double vectors) of
// coefficient type vt and SELL layout c16 keeps resident.
int sellKernelOccupancy(DType vt, bool c16);

// SpMV autotuner: times every candidate launch geometry `reps` times on the
// matrix's stream and keeps the fastest for vectors of type t. The results
// of gr_spmv do not depend on the geometry.
SpmvTuning tuneSpmv(DeviceMatrix& A, DType t, int reps);
// Mean device time (ms) of y = A x with the current geometry over `reps`
// launches, each timed alone on the matrix's stream (L2 flushed first when
// flushL2).
float timeSpmv(DeviceMatrix& A, const void* x, void* y, DType t, int reps, bool flushL2);

// r = b - A x in inter (reference CRSMatrix::residual); optionally
// accumulates a norm of r into normOut (device double) when normKind >= 0.
// For a batch matrix every system's norm goes to normOut[system], reduced
// over the blocks and in the order a solve of that system alone uses.
void launchResidual(DeviceMatrix& A, const void* x, DType xt, const void* b, DType bt, void* r,
                    DType rt, DType inter, int normKind, double* normOut, cudaStream_t s);

// Norm of the first n entries of x (same geometry as a matrix of n rows).
void launchNormN(DeviceMatrix& A, const void* x, i64 n, DType t, int normKind, double* out, cudaStream_t s);

// Norm of a tile-order vector, FP64 accumulation. normKind: gr_norm.
void launchNorm(DeviceMatrix& A, const void* x, DType t, int normKind, double* out,
                cudaStream_t s);

void launchPermute(DeviceMatrix& A, const void* src, void* dst, DType t, bool toTileOrder,
                   cudaStream_t s);

// Norms of `count` vectors through a static device scratch, allocating
// nothing (gr_vector_norms_noalloc).
void launchNormsNoAlloc(const void* x, i64 n, i64 count, i64 ld, DType t, int normKind, double* out,
                        cudaStream_t s);

}  // namespace gr

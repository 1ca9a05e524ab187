// Level schedules for the tile-local sweeps (ILU forward / backward
// substitution, Gauss-Seidel) and their upload. See LevelSchedule in
// device.hpp for the layout.
//
// The reference runs these sweeps sequentially per tile on the CPU target and
// over the same level sets ("colours", CRSHostMatrix.cpp:527-675) on the IPU
// (ilu/Solver.cpp:444-522). Rows of one level depend only on rows of earlier
// levels, so processing the levels in order with the rows of a level in
// parallel performs exactly the sequential sweep's operations.
#include <algorithm>
#include <cstring>

#include "device.hpp"
#include "krylov.hpp"

namespace gr {

namespace {

struct TileSched {
  std::vector<i32> lvlRows;   // rows per level
  std::vector<i64> lvlSlots;  // slots per level
  std::vector<i32> rows;      // tile-order rows, level-major
  std::vector<i32> col;       // slots
  std::vector<i32> src;
};

// Entries of tile-order row p (tile-local index il, tile rows nRows) that a
// sweep of the given kind reads, in the order the reference reads them.
void rowEntries(const HostMatrix& H, SweepEntries kind, i64 p, i64 il, i64 nRows, std::vector<i64>& out) {
  out.clear();
  const i64 b = H.rowPtr[p], e = H.rowPtr[p + 1];
  switch (kind) {
    case SweepEntries::Lower:  // ilu/Solver.cpp:391-403, ascending, stop at the diagonal
      for (i64 k = b; k < e; ++k) {
        i64 j = H.colLocal[k];
        if (il < j || j >= nRows) break;
        out.push_back(k);
      }
      break;
    case SweepEntries::UpperDesc:  // ilu/Solver.cpp:424-436, descending, halo skipped
      for (i64 k = e - 1; k >= b; --k) {
        i64 j = H.colLocal[k];
        if (j < il) break;
        if (j >= nRows) continue;
        out.push_back(k);
      }
      break;
    case SweepEntries::All:  // gauss-seidel/Solver.cpp:76-79, every entry in order
      for (i64 k = b; k < e; ++k) out.push_back(k);
      break;
  }
}

}  // namespace

LevelSchedule& DeviceMatrix::schedule(SweepEntries kind) {
  std::unique_ptr<LevelSchedule>& slot =
      kind == SweepEntries::Lower ? lowerSched : (kind == SweepEntries::UpperDesc ? upperSched : gsSched);
  if (slot) return *slot;
  const HostMatrix& H = *host;
  const bool upper = kind == SweepEntries::UpperDesc;
  std::vector<TileSched> ts(H.P);
  parallelFor(H.P, [&](i64 T) {
    TileSched& s = ts[T];
    const i64 base = H.tileStart[T];
    const i64 nRows = H.tileStart[T + 1] - base;
    const i32 nL = upper ? H.nUpperLevels[T] : H.nLowerLevels[T];
    const std::vector<i32>& lev = upper ? H.upperLevel : H.lowerLevel;
    std::vector<std::vector<i64>> byLevel(nL);
    for (i64 i = 0; i < nRows; ++i) byLevel[lev[base + i]].push_back(i);
    std::vector<i64> ent;
    for (i32 l = 0; l < nL; ++l) {
      const auto& rows = byLevel[l];
      const i64 k = static_cast<i64>(rows.size());
      i64 maxE = 0;
      for (i64 il : rows) {
        rowEntries(H, kind, base + il, il, nRows, ent);
        maxE = std::max<i64>(maxE, static_cast<i64>(ent.size()));
      }
      const size_t off = s.col.size();
      s.col.resize(off + k * maxE, -1);
      s.src.resize(off + k * maxE, -1);
      for (i64 q = 0; q < k; ++q) {
        const i64 il = rows[q];
        s.rows.push_back(static_cast<i32>(base + il));
        rowEntries(H, kind, base + il, il, nRows, ent);
        for (size_t e = 0; e < ent.size(); ++e) {
          s.col[off + e * k + q] = H.colPerm[ent[e]];
          s.src[off + e * k + q] = static_cast<i32>(ent[e]);
        }
      }
      s.lvlRows.push_back(static_cast<i32>(k));
      s.lvlSlots.push_back(k * maxE);
    }
  });
  auto S = std::make_unique<LevelSchedule>();
  std::vector<i32> tileLvlStart(H.P + 1, 0), lvlRowStart(1, 0);
  std::vector<i64> lvlSlotStart(1, 0);
  std::vector<i32> rows, col, src;
  i32 maxRows = 0;
  for (i32 T = 0; T < H.P; ++T) {
    const TileSched& s = ts[T];
    tileLvlStart[T + 1] = tileLvlStart[T] + static_cast<i32>(s.lvlRows.size());
    for (size_t l = 0; l < s.lvlRows.size(); ++l) {
      lvlRowStart.push_back(lvlRowStart.back() + s.lvlRows[l]);
      lvlSlotStart.push_back(lvlSlotStart.back() + s.lvlSlots[l]);
      maxRows = std::max(maxRows, s.lvlRows[l]);
    }
    rows.insert(rows.end(), s.rows.begin(), s.rows.end());
    col.insert(col.end(), s.col.begin(), s.col.end());
    src.insert(src.end(), s.src.begin(), s.src.end());
  }
  if (lvlSlotStart.back() >= (i64(1) << 31)) fail(GR_EUNSUPPORTED, "level schedule exceeds 2^31 slots");
  S->numLevels = tileLvlStart[H.P];
  S->maxLevelRows = maxRows;
  S->slots = lvlSlotStart.back();
  S->tileLvlStart.upload(tileLvlStart);
  S->lvlRowStart.upload(lvlRowStart);
  S->lvlSlotStart.upload(lvlSlotStart);
  S->rows.upload(rows);
  S->col.upload(col);
  S->src.upload(src);
  slot = std::move(S);
  return *slot;
}

// ---------------------------------------------------------------------------
// ILU application stream (see SweepStream in device.hpp).
namespace {

inline i64 pad16(i64 b) { return (b + 15) & ~i64(15); }

struct TileBytes {
  std::vector<uint8_t> bytes;
  std::vector<std::pair<i64, i32>> vals;  // (byte offset in tile stream, CRS source or -1)
  std::vector<std::pair<i64, i32>> invs;  // (byte offset, tile-order row)
  i64 maxLevel = 0;
  i64 maxSpan = 0;
  std::vector<i64> levelStart;  // byte offset of every level header, then the end
  std::vector<int4> table;      // {offset, k, E, hasInv} per level
};

void putInt4(std::vector<uint8_t>& b, i32 a, i32 c, i32 d, i32 e) {
  const i32 v[4] = {a, c, d, e};
  const size_t o = b.size();
  b.resize(o + 16);
  std::memcpy(b.data() + o, v, 16);
}

}  // namespace

HostStream buildIluStream(const HostMatrix& H, bool dilu, DType vt) {
  const i64 vs = static_cast<i64>(dtypeSize(vt));
  std::vector<TileBytes> tb(H.P);
  parallelFor(H.P, [&](i64 T) {
    TileBytes& t = tb[T];
    const i64 base = H.tileStart[T];
    const i64 nRows = H.tileStart[T + 1] - base;
    putInt4(t.bytes, H.nLowerLevels[T], H.nUpperLevels[T], 0, 0);
    std::vector<i64> ent;
    for (int sweep = 0; sweep < 2; ++sweep) {
      const bool upper = sweep == 1;
      const SweepEntries kind = upper ? SweepEntries::UpperDesc : SweepEntries::Lower;
      const i32 nL = upper ? H.nUpperLevels[T] : H.nLowerLevels[T];
      const std::vector<i32>& lev = upper ? H.upperLevel : H.lowerLevel;
      std::vector<std::vector<i64>> byLevel(nL);
      for (i64 i = 0; i < nRows; ++i) byLevel[lev[base + i]].push_back(i);
      const bool hasInv = upper || dilu;
      for (i32 l = 0; l < nL; ++l) {
        const auto& rows = byLevel[l];
        const i64 k = static_cast<i64>(rows.size());
        i64 E = 0;
        for (i64 il : rows) {
          rowEntries(H, kind, base + il, il, nRows, ent);
          E = std::max<i64>(E, static_cast<i64>(ent.size()));
        }
        const i64 start = static_cast<i64>(t.bytes.size());
        t.levelStart.push_back(start);
        t.table.push_back(make_int4(static_cast<int>(start), static_cast<int>(k), static_cast<int>(E), hasInv ? 1 : 0));
        putInt4(t.bytes, static_cast<i32>(k), static_cast<i32>(E), hasInv ? 1 : 0, 0);
        const i64 rowsOff = static_cast<i64>(t.bytes.size());
        const i64 invOff = rowsOff + pad16(4 * k);
        const i64 colsOff = invOff + (hasInv ? pad16(vs * k) : 0);
        const i64 valsOff = colsOff + pad16(4 * E * k);
        const i64 end = valsOff + pad16(vs * E * k);
        t.bytes.resize(end, 0);
        std::vector<i32> cols(E * k, -1);
        for (i64 q = 0; q < k; ++q) {
          const i64 il = rows[q];
          const i32 r32 = static_cast<i32>(il);
          std::memcpy(t.bytes.data() + rowsOff + 4 * q, &r32, 4);
          if (hasInv) t.invs.emplace_back(invOff + vs * q, static_cast<i32>(base + il));
          rowEntries(H, kind, base + il, il, nRows, ent);
          for (i64 e = 0; e < E; ++e) {
            const bool real = e < static_cast<i64>(ent.size());
            cols[e * k + q] = real ? H.colLocal[ent[e]] : -1;
            t.vals.emplace_back(valsOff + vs * (e * k + q), real ? static_cast<i32>(ent[e]) : -1);
          }
        }
        std::memcpy(t.bytes.data() + colsOff, cols.data(), 4 * E * k);
        t.maxLevel = std::max(t.maxLevel, end - start);
      }
    }
    t.levelStart.push_back(static_cast<i64>(t.bytes.size()));
    // Spans: tile header through level 0, then level l through level l + 1.
    const size_t L = t.levelStart.size() - 1;
    if (L > 0) t.maxSpan = t.levelStart[1];
    for (size_t l = 0; l + 1 < L; ++l) t.maxSpan = std::max(t.maxSpan, t.levelStart[l + 2] - t.levelStart[l]);
    if (L == 1) t.maxSpan = std::max(t.maxSpan, t.levelStart[1] - t.levelStart[0]);
    t.bytes.resize(pad16(static_cast<i64>(t.bytes.size())), 0);
  });
  HostStream S;
  S.tileOffset.assign(H.P + 1, 0);
  i64 nVal = 0, nInv = 0;
  for (i32 T = 0; T < H.P; ++T) {
    S.tileOffset[T + 1] = S.tileOffset[T] + static_cast<i64>(tb[T].bytes.size());
    S.maxLevelBytes = std::max(S.maxLevelBytes, tb[T].maxLevel);
    S.maxSpanBytes = std::max(S.maxSpanBytes, tb[T].maxSpan);
    S.maxTileLevels = std::max<i32>(S.maxTileLevels, static_cast<i32>(tb[T].table.size()));
    for (const int4& d : tb[T].table) {
      S.maxLevelRows = std::max<i32>(S.maxLevelRows, d.y);
      S.maxEntries = std::max<i32>(S.maxEntries, d.z);
    }
    nVal += static_cast<i64>(tb[T].vals.size());
    nInv += static_cast<i64>(tb[T].invs.size());
  }
  S.tileLevel.assign(H.P + 1, 0);
  for (i32 T = 0; T < H.P; ++T) {
    S.tileLevel[T + 1] = S.tileLevel[T] + static_cast<i32>(tb[T].table.size());
    S.levelTable.insert(S.levelTable.end(), tb[T].table.begin(), tb[T].table.end());
  }
  const i64 total = S.tileOffset[H.P];
  if (total / vs >= (i64(1) << 31)) fail(GR_EUNSUPPORTED, "ILU stream exceeds 2^31 elements");
  S.bytes.resize(total);
  S.valPos.resize(nVal);
  S.valSrc.resize(nVal);
  S.invPos.resize(nInv);
  S.invSrc.resize(nInv);
  std::vector<i64> vOff(H.P + 1, 0), iOff(H.P + 1, 0);
  for (i32 T = 0; T < H.P; ++T) {
    vOff[T + 1] = vOff[T] + static_cast<i64>(tb[T].vals.size());
    iOff[T + 1] = iOff[T] + static_cast<i64>(tb[T].invs.size());
  }
  parallelFor(H.P, [&](i64 T) {
    const i64 off = S.tileOffset[T];
    std::memcpy(S.bytes.data() + off, tb[T].bytes.data(), tb[T].bytes.size());
    for (size_t i = 0; i < tb[T].vals.size(); ++i) {
      S.valPos[vOff[T] + i] = static_cast<i32>((off + tb[T].vals[i].first) / vs);
      S.valSrc[vOff[T] + i] = tb[T].vals[i].second;
    }
    for (size_t i = 0; i < tb[T].invs.size(); ++i) {
      S.invPos[iOff[T] + i] = static_cast<i32>((off + tb[T].invs[i].first) / vs);
      S.invSrc[iOff[T] + i] = tb[T].invs[i].second;
    }
  });
  return S;
}

int ringLog2ForLevel(i64 maxLevelBytes) {
  // The largest level plus one partially consumed chunk must fit in the
  // ring: ring >= maxLevel * R / (R - 1) + 16.
  const i64 need = maxLevelBytes * kRingChunksHost / (kRingChunksHost - 1) + 16;
  int lg = 13;  // 8 KB minimum
  while ((i64(1) << lg) < need) ++lg;
  return lg;
}

// Replays the streamed kernel's consumption of every tile's stream on the
// host: headers and segment offsets, index ranges, the level order each
// entry depends on, and that every chunk a level needs has been issued under
// the producer's refill rule: before waiting for level l + 1, thread 0 has
// issued every chunk below start(l) / C + R (start(l) = byte offset of level
// l's header); before the loop, chunks 0 .. R - 1. Throws on the first
// violation.
void checkIluStream(const HostMatrix& H, const HostStream& S, bool dilu, DType vt, int ringLog2) {
  const i64 vs = static_cast<i64>(dtypeSize(vt));
  const i64 ring = i64(1) << ringLog2, C = ring / kRingChunksHost;
  parallelFor(H.P, [&](i64 T) {
    const uint8_t* g = S.bytes.data() + S.tileOffset[T];
    const i64 len = S.tileOffset[T + 1] - S.tileOffset[T];
    const i64 base = H.tileStart[T];
    const i64 nRows = H.tileStart[T + 1] - base;
    auto bad = [&](const std::string& what) {
      fail(GR_EINVAL, "ILU stream check failed in tile " + std::to_string(T) + ": " + what);
    };
    if (len % 16 != 0 || S.tileOffset[T] % 16 != 0) bad("misaligned tile stream");
    const i64 total = (len + C - 1) / C;
    i64 issued = std::min<i64>(total, kRingChunksHost);
    auto needChunks = [&](i64 endByte) {
      const i64 need = (endByte + C - 1) / C;
      if (need > issued) bad("level needs chunk " + std::to_string(need - 1) + " before it is issued");
      if (endByte > len) bad("read past the end of the stream");
    };
    auto rd = [&](i64 o) {
      i32 v;
      std::memcpy(&v, g + o, 4);
      return v;
    };
    needChunks(16);
    const i32 nL = rd(0), nU = rd(4);
    if (nL != H.nLowerLevels[T] || nU != H.nUpperLevels[T]) bad("level counts");
    std::vector<i32> doneLower(nRows, -1), doneUpper(nRows, -1);
    i64 off = 16, prevStart = -1;
    for (i32 lv = 0; lv < nL + nU; ++lv) {
      const bool upper = lv >= nL;
      if (lv > 0) issued = std::min<i64>(total, prevStart / C + kRingChunksHost);
      needChunks(off + 16);
      const i64 k = rd(off), E = rd(off + 4);
      const bool hasInv = rd(off + 8) != 0;
      if (k <= 0 || E < 0) bad("empty level");
      if (hasInv != (upper || dilu)) bad("inverse-diagonal flag");
      if (S.tileLevel[T + 1] - S.tileLevel[T] != nL + nU) bad("level table size");
      const int4 d = S.levelTable[S.tileLevel[T] + lv];
      if (d.x != off || d.y != k || d.z != E || d.w != (hasInv ? 1 : 0)) bad("level table entry");
      const i64 rowsOff = off + 16;
      const i64 invOff = rowsOff + pad16(4 * k);
      const i64 colsOff = invOff + (hasInv ? pad16(vs * k) : 0);
      const i64 valsOff = colsOff + pad16(4 * E * k);
      const i64 end = valsOff + pad16(vs * E * k);
      needChunks(end);
      for (i64 q = 0; q < k; ++q) {
        const i32 il = rd(rowsOff + 4 * q);
        if (il < 0 || il >= nRows) bad("row id out of range");
        std::vector<i32>& done = upper ? doneUpper : doneLower;
        if (done[il] >= 0) bad("row listed twice in one sweep");
        bool padding = false;
        for (i64 e = 0; e < E; ++e) {
          const i32 c = rd(colsOff + 4 * (e * k + q));
          if (c < 0) {
            padding = true;
            continue;
          }
          if (padding) bad("column after padding");
          if (c >= nRows) bad("column out of range");
          if (!upper && !(c < il)) bad("forward entry not below the diagonal");
          if (upper && !(c > il)) bad("backward entry not above the diagonal");
          if (done[c] < 0) bad("entry read before its row is computed");
        }
      }
      for (i64 q = 0; q < k; ++q) (upper ? doneUpper : doneLower)[rd(rowsOff + 4 * q)] = lv;
      prevStart = off;
      off = end;
    }
    if (off != len) bad("stream length does not match its levels");
    for (i64 i = 0; i < nRows; ++i)
      if (doneLower[i] < 0 || doneUpper[i] < 0) bad("row missing from a sweep");
  });
}

SweepStream& DeviceMatrix::iluSweepStream(bool dilu) {
  std::unique_ptr<SweepStream>& slot = iluStream[dilu ? 1 : 0];
  if (slot) return *slot;
  HostStream H = buildIluStream(*host, dilu, vt);
  auto S = std::make_unique<SweepStream>();
  S->dilu = dilu;
  S->bytes = static_cast<i64>(H.bytes.size());
  S->maxLevelBytes = H.maxLevelBytes;
  S->maxSpanBytes = H.maxSpanBytes;
  S->levelTable.upload(H.levelTable);
  S->tileLevel.upload(H.tileLevel);
  S->numLevels = static_cast<i64>(H.levelTable.size());
  S->maxTileLevels = H.maxTileLevels;
  S->maxLevelRows = H.maxLevelRows;
  S->maxEntries = H.maxEntries;
  S->nVal = static_cast<i64>(H.valPos.size());
  S->nInv = static_cast<i64>(H.invPos.size());
  S->tileOffset.upload(H.tileOffset);
  S->templ.upload(H.bytes);
  S->valPos.upload(H.valPos);
  S->valSrc.upload(H.valSrc);
  S->invPos.upload(H.invPos);
  S->invSrc.upload(H.invSrc);
  slot = std::move(S);
  return *slot;
}

}  // namespace gr

// ---------------------------------------------------------------------------
// Host-scheduled level ring (kernels_ring.cu).
namespace gr {

namespace {
struct TileRing {
  std::vector<uint8_t> bytes;
  std::vector<int4> meta;
  std::vector<std::pair<i64, i32>> vals;  // (byte offset of the value, CRS source)
  std::vector<std::pair<i64, i32>> invs;  // (byte offset, tile-order row)
  std::vector<i64> size;
  i64 maxLevel = 0;
};

inline bool overlaps(i64 a, i64 sa, i64 b, i64 sb) { return a < b + sb && b < a + sa; }
}  // namespace

HostRing buildLevelRing(const HostMatrix& H, bool dilu, DType vt, i64 ringBytes, i32 group,
                        const RingBudget& budget, bool allowCompact, RingKind kind, bool records) {
  const i64 vs = static_cast<i64>(dtypeSize(vt));
  const i64 entSize = vs == 4 ? 8 : 16;
  const bool gs = kind != RingKind::Ilu;
  if (group < 1) fail(GR_EINVAL, "tiles per block must be at least 1");
  if (gs && group != 1) fail(GR_EINVAL, "Gauss-Seidel rings run one tile per block");
  // A block runs `group` consecutive tiles in lockstep: level l of the block
  // is level l of each of its tiles (the tiles are independent, so their
  // rows never reference one another), rows numbered from the block's first
  // row.
  const i32 NG = (H.P + group - 1) / group;
  i64 maxGroupRows = 0;
  for (i32 G = 0; G < NG; ++G)
    maxGroupRows = std::max<i64>(maxGroupRows, H.tileStart[std::min<i32>(H.P, (G + 1) * group)] - H.tileStart[G * group]);
  // Gauss-Seidel: x slots per tile (this sweep's values, the sweep-start
  // values, the halo and the zero slot) and the halo cells' tile-order
  // indices.
  i64 maxGsSlots = 0;
  std::vector<i32> haloStart, haloSrc;
  // In place: every in-tile entry above the diagonal lies in a later level
  // than its row (a lexicographically numbered box of a 7-point grid, for
  // one), so when a row is updated its upper neighbours still hold their
  // start values and the sweep needs no copy of them.
  bool inPlace = gs;
  if (gs && kind == RingKind::GaussSeidel) {
    std::atomic<bool> ok{true};
    parallelFor(H.P, [&](i64 T) {
      const i64 base = H.tileStart[T], nRows = H.tileStart[T + 1] - base;
      for (i64 r = 0; r < nRows && ok.load(std::memory_order_relaxed); ++r)
        for (i64 k = H.rowPtr[base + r]; k < H.rowPtr[base + r + 1]; ++k) {
          const i64 lc = H.colLocal[k];
          if (lc > r && lc < nRows && H.lowerLevel[base + lc] <= H.lowerLevel[base + r]) {
            ok = false;
            break;
          }
        }
    });
    inPlace = ok;
  }
  if (gs) {
    haloStart.assign(H.P + 1, 0);
    for (i32 T = 0; T < H.P; ++T) {
      haloStart[T + 1] = haloStart[T] + static_cast<i32>(H.tiles[T].nHalo);
      maxGsSlots = std::max<i64>(maxGsSlots, (inPlace ? 1 : 2) * H.tiles[T].rows() + H.tiles[T].nHalo + 1);
    }
    haloSrc.assign(haloStart[H.P], -1);
    parallelFor(H.P, [&](i64 T) {
      const i64 base = H.tileStart[T], nRows = H.tileStart[T + 1] - base;
      for (i64 k = H.rowPtr[base]; k < H.rowPtr[base + nRows]; ++k)
        if (H.colLocal[k] >= nRows) haloSrc[haloStart[T] + H.colLocal[k] - nRows] = H.colPerm[k];
    });
    for (i32 v : haloSrc)
      if (v < 0) fail(GR_EINVAL, "Gauss-Seidel ring: a halo cell no entry reads");
  }
  const bool compact = allowCompact && (gs ? maxGsSlots <= kRingCompactRows : maxGroupRows + 1 <= kRingCompactRows);
  std::vector<TileRing> tr(NG);
  parallelFor(NG, [&](i64 G) {
    TileRing& t = tr[G];
    const i32 T0 = static_cast<i32>(G) * group, T1 = std::min<i32>(H.P, T0 + group);
    const i64 gBase = H.tileStart[T0];
    const i64 gRows = H.tileStart[T1] - gBase;
    std::vector<i64> ent;
    const i64 zeroSlot = gs ? (inPlace ? 1 : 2) * gRows + H.tiles[T0].nHalo : gRows;
    const i64 startBase = inPlace ? 0 : gRows;  // Gauss-Seidel: where start values live
    for (int sweep = 0; sweep < (gs ? 1 : 2); ++sweep) {
      const bool upper = sweep == 1;
      const SweepEntries ekind = gs ? (kind == RingKind::GaussSeidelLower ? SweepEntries::Lower : SweepEntries::All)
                                    : (upper ? SweepEntries::UpperDesc : SweepEntries::Lower);
      const std::vector<i32>& lev = upper ? H.upperLevel : H.lowerLevel;
      i32 nLv = 0;
      for (i32 T = T0; T < T1; ++T) nLv = std::max(nLv, upper ? H.nUpperLevels[T] : H.nLowerLevels[T]);
      // (block-local row, tile) per level
      std::vector<std::vector<std::pair<i64, i32>>> byLevel(nLv);
      for (i32 T = T0; T < T1; ++T)
        for (i64 p = H.tileStart[T]; p < H.tileStart[T + 1]; ++p) byLevel[lev[p]].emplace_back(p - gBase, T);
      const bool hasInv = gs || upper || dilu;  // Gauss-Seidel: the diagonal
      for (i32 l = 0; l < nLv; ++l) {
        const auto& rows = byLevel[l];
        const i64 k = static_cast<i64>(rows.size());
        i64 E = 0;
        for (const auto& [gl, T] : rows) {
          const i64 tb = H.tileStart[T] - gBase;
          rowEntries(H, ekind, gBase + gl, gl - tb, H.tileStart[T + 1] - H.tileStart[T], ent);
          E = std::max<i64>(E, static_cast<i64>(ent.size()));
        }
        if (E >= (i64(1) << kRingEBits) || k >= (i64(1) << 31) || entSize * E * k >= (i64(1) << 31))
          fail(GR_EUNSUPPORTED, "ILU level too large for the ring kernel");
        const bool rec = records && ringRecordLevel(static_cast<uint32_t>(E), static_cast<uint32_t>(vs), compact);
        const RingLevelLayout lay = ringLevelLayout(static_cast<uint32_t>(k), static_cast<uint32_t>(E), hasInv,
                                                    static_cast<uint32_t>(vs), compact, rec);
        const i64 S = lay.bytes;
        const i64 start = static_cast<i64>(t.bytes.size());
        t.bytes.resize(start + S, 0);
        if (rec) {
          // Record level: {v0, v1, v2, c0 | c1 << 16} per row, then
          // {c2 | row << 16} (and the inverse diagonal) per row.
          const i64 recB = hasInv ? 8 : 4;
          for (i64 q = 0; q < k; ++q) {
            const auto [gl, T] = rows[q];
            const i64 tb = H.tileStart[T] - gBase;
            rowEntries(H, ekind, gBase + gl, gl - tb, H.tileStart[T + 1] - H.tileStart[T], ent);
            uint32_t c[3];
            for (int e = 0; e < 3; ++e) {
              const bool real = e < static_cast<int>(ent.size());
              i64 col = zeroSlot;
              if (real) {
                const i64 lc = H.colLocal[ent[e]];
                col = gs ? (lc < gl ? lc : startBase + lc) : lc + tb;
                t.vals.emplace_back(start + 16 * q + 4 * e, static_cast<i32>(ent[e]));
              }
              c[e] = static_cast<uint32_t>(col);
            }
            const uint32_t w01 = c[0] | (c[1] << 16), w2 = c[2] | (static_cast<uint32_t>(gl) << 16);
            std::memcpy(t.bytes.data() + start + 16 * q + 12, &w01, 4);
            std::memcpy(t.bytes.data() + start + lay.ents + recB * q, &w2, 4);
            if (hasInv) t.invs.emplace_back(start + lay.ents + recB * q + 4, static_cast<i32>(gBase + gl));
          }
          t.meta.push_back(make_int4(static_cast<int>(k), static_cast<int>(static_cast<uint32_t>(E) |
                                                                              (upper ? kRingUpperBit : 0u) |
                                                                              kRingRecordBit),
                                     0, -1));
          t.size.push_back(S);
          t.maxLevel = std::max(t.maxLevel, S);
          continue;
        }
        for (i64 q = 0; q < k; ++q) {
          const auto [gl, T] = rows[q];
          const i64 tb = H.tileStart[T] - gBase;
          if (compact) {
            const uint16_t r16 = static_cast<uint16_t>(gl);
            std::memcpy(t.bytes.data() + start + 2 * q, &r16, 2);
          } else {
            const i32 r32 = static_cast<i32>(gl);
            std::memcpy(t.bytes.data() + start + 4 * q, &r32, 4);
          }
          if (hasInv) t.invs.emplace_back(start + lay.inv + vs * q, static_cast<i32>(gBase + gl));
          rowEntries(H, ekind, gBase + gl, gl - tb, H.tileStart[T + 1] - H.tileStart[T], ent);
          for (i64 e = 0; e < E; ++e) {
            const bool real = e < static_cast<i64>(ent.size());
            i32 col = static_cast<i32>(zeroSlot);
            if (real) {
              const i64 lc = H.colLocal[ent[e]];
              col = static_cast<i32>(gs ? (lc < gl ? lc : startBase + lc) : lc + tb);
            }
            if (compact) {
              const uint16_t c16 = static_cast<uint16_t>(col);
              std::memcpy(t.bytes.data() + start + lay.ents + 2 * (e * k + q), &c16, 2);
              if (real) t.vals.emplace_back(start + lay.vals + vs * (e * k + q), static_cast<i32>(ent[e]));
            } else {
              const i64 pos = start + lay.ents + entSize * (e * k + q);
              std::memcpy(t.bytes.data() + pos, &col, 4);
              if (real) t.vals.emplace_back(pos + (vs == 4 ? 4 : 8), static_cast<i32>(ent[e]));
            }
          }
        }
        t.meta.push_back(make_int4(static_cast<int>(k), static_cast<int>(E) | (upper ? kRingUpperBit : 0), 0, -1));
        t.size.push_back(S);
        t.maxLevel = std::max(t.maxLevel, S);
      }
    }
  });
  HostRing R;
  for (const TileRing& t : tr) R.maxLevelBytes = std::max(R.maxLevelBytes, t.maxLevel);
  // Ring placement. Level l goes to the offset, among the ring's two ends and
  // the ends and starts of the levels of the last kRingBarriers, whose copy
  // can be issued earliest: after the most recent earlier level whose block
  // it overlaps, the level that last used its completion barrier, and the
  // previous level's copy. Offsets that leave level l + 1 a place beside it
  // (at either end of the ring or right after it) come first, so that any
  // ring of at least two of the largest levels places. Ties go to the offset
  // right after level l - 1, then to the one found first. Placement fails
  // when some level would have to wait for the level right before it.
  auto place = [&](i64 ring) {
    std::atomic<bool> ok{true};
    parallelFor(NG, [&](i64 T) {
      TileRing& t = tr[T];
      const i64 L = static_cast<i64>(t.size.size());
      std::vector<i64> off(L);
      i64 prevIa = -1;
      for (i64 l = 0; l < L && ok; ++l) {
        const i64 S = t.size[l];
        if (S > ring || S >= (i64(1) << (32 - kRingOffBits + 4))) { ok = false; return; }
        const i64 floorIa = std::max<i64>(prevIa, l - kRingBarriers);
        // issueAfter for offset c: the most recent overlapping level above
        // floorIa, else floorIa.
        auto issueAfter = [&](i64 c) {
          for (i64 j = l - 1; j > floorIa; --j)
            if (overlaps(off[j], t.size[j], c, S)) return j;
          return floorIa;
        };
        const i64 Sn = l + 1 < L ? t.size[l + 1] : 0;
        i64 best = -1, bestIa = 0;
        bool bestRoom = false;
        auto consider = [&](i64 c) {
          if (c < 0 || c + S > ring || c % 16 != 0) return;
          const i64 ia = issueAfter(c);
          const bool room = Sn == 0 || c >= Sn || c + S + Sn <= ring;
          if (best < 0 || (room && !bestRoom) || (room == bestRoom && ia < bestIa)) {
            best = c;
            bestIa = ia;
            bestRoom = room;
          }
        };
        if (l > 0) consider(off[l - 1] + t.size[l - 1]);
        consider(0);
        consider((ring - S) / 16 * 16);
        for (i64 j = l - 1; j >= 0 && j >= l - kRingBarriers; --j) {
          consider(off[j] + t.size[j]);
          consider(off[j] - S);
        }
        if (best < 0 || (l >= 1 && bestIa > l - 2)) { ok = false; return; }
        off[l] = best;
        t.meta[l].z = static_cast<int>(best);
        t.meta[l].w = static_cast<int>(bestIa);
        prevIa = bestIa;
      }
    });
    return ok.load();
  };
  i32 maxLevels = 0;
  for (const TileRing& t : tr) maxLevels = std::max<i32>(maxLevels, static_cast<i32>(t.size.size()));
  if (ringBytes > 0) {
    R.ringBytes = pad16(ringBytes);
    if (!place(R.ringBytes))
      fail(GR_EINVAL, "ILU level ring of " + std::to_string(R.ringBytes) + " bytes is too small for this matrix's levels");
  } else {
    // Default: among the ring sizes from twice the largest level up to
    // max(16 KB, 4 x the largest level), in steps of 256 bytes (or 1/16 of
    // the largest level), one that places and runs all blocks in the fewest
    // waves (blocks resident per SM from the budget); the largest such, as a
    // larger ring lets copies run further ahead.
    const i64 fixed = ringFixedSmemSlots(maxLevels, gs ? maxGsSlots + maxGroupRows : maxGroupRows + 1, vs) +
                      budget.reservedPerBlock;
    const i64 lo = std::max<i64>(256, pad16(2 * R.maxLevelBytes));
    const i64 hi = std::max<i64>(std::max<i64>(16384, pad16(4 * R.maxLevelBytes)), lo);
    const i64 step = std::max<i64>(256, pad16(R.maxLevelBytes / 16));
    // Waves depend only on the size, so the sizes are tried best first
    // (fewest waves, then largest); the first that places is taken, which
    // usually costs one or two placement passes.
    auto wavesOf = [&](i64 r) {
      const i64 perSM = std::min<i64>(budget.maxBlocksPerSM, budget.smemPerSM / (fixed + r));
      const i64 slots = std::max<i64>(1, perSM) * std::max<i32>(1, budget.numSMs);
      return perSM > 0 ? (NG + slots - 1) / slots : (i64(1) << 40);
    };
    std::vector<std::pair<i64, i64>> order;  // (waves, -size)
    for (i64 r = lo; r < hi; r += step) order.emplace_back(wavesOf(r), -r);
    order.emplace_back(wavesOf(hi), -hi);
    std::sort(order.begin(), order.end());
    i64 bestRing = -1;
    for (const auto& [w, negR] : order) {
      if (place(-negR)) {
        bestRing = -negR;
        break;
      }
    }
    for (i64 r = hi + step; bestRing < 0 && r < (i64(1) << kRingOffBits); r += step)
      if (place(r)) bestRing = r;
    if (bestRing < 0) fail(GR_EUNSUPPORTED, "ILU level ring too large");
    R.ringBytes = bestRing;  // the last placement pass was this size's
  }
  if (R.ringBytes > (i64(1) << kRingOffBits)) fail(GR_EUNSUPPORTED, "ILU level ring too large");
  R.group = group;
  R.compact = compact;
  R.kind = kind;
  R.maxXSlots = gs ? maxGsSlots + maxGroupRows : maxGroupRows + 1;
  R.gsInPlace = gs && inPlace;
  R.haloStart = std::move(haloStart);
  R.haloSrc = std::move(haloSrc);
  R.tileOffset.assign(NG + 1, 0);
  R.tileLevel.assign(NG + 1, 0);
  R.groupStart.assign(NG + 1, 0);
  for (i32 G = 0; G <= NG; ++G) R.groupStart[G] = static_cast<i32>(H.tileStart[std::min<i32>(H.P, G * group)]);
  for (i32 G = 0; G < NG; ++G) R.maxGroupRows = std::max<i64>(R.maxGroupRows, R.groupStart[G + 1] - R.groupStart[G]);
  i64 nVal = 0, nInv = 0;
  for (i32 T = 0; T < NG; ++T) {
    R.tileOffset[T + 1] = R.tileOffset[T] + static_cast<i64>(tr[T].bytes.size());
    R.tileLevel[T + 1] = R.tileLevel[T] + static_cast<i32>(tr[T].size.size());
    R.maxTileLevels = std::max<i32>(R.maxTileLevels, static_cast<i32>(tr[T].size.size()));
    nVal += static_cast<i64>(tr[T].vals.size());
    nInv += static_cast<i64>(tr[T].invs.size());
  }
  const i64 total = R.tileOffset[NG];
  if (total / vs >= (i64(1) << 31)) fail(GR_EUNSUPPORTED, "ILU level ring stream exceeds 2^31 elements");
  R.bytes.resize(total);
  R.meta.resize(static_cast<size_t>(R.tileLevel[NG]));
  R.valPos.resize(nVal);
  R.valSrc.resize(nVal);
  R.invPos.resize(nInv);
  R.invSrc.resize(nInv);
  std::vector<i64> vOff(NG + 1, 0), iOff(NG + 1, 0);
  for (i32 T = 0; T < NG; ++T) {
    vOff[T + 1] = vOff[T] + static_cast<i64>(tr[T].vals.size());
    iOff[T + 1] = iOff[T] + static_cast<i64>(tr[T].invs.size());
  }
  parallelFor(NG, [&](i64 T) {
    const i64 off = R.tileOffset[T];
    std::memcpy(R.bytes.data() + off, tr[T].bytes.data(), tr[T].bytes.size());
    // Pack the placed levels (RingLevelCode): E, entries offset and sweep in
    // y; ring offset and block size in z.
    for (size_t l = 0; l < tr[T].meta.size(); ++l) {
      int4 m = tr[T].meta[l];
      const bool upper = (m.y & kRingUpperBit) != 0;
      const bool rec = (static_cast<uint32_t>(m.y) & kRingRecordBit) != 0;
      const uint32_t E = static_cast<uint32_t>(m.y) & ((1u << kRingEBits) - 1);
      const RingLevelLayout lay = ringLevelLayout(static_cast<uint32_t>(m.x), E, gs || upper || dilu,
                                                  static_cast<uint32_t>(vs), compact, rec);
      m.y = static_cast<int>(E | ((lay.ents >> 4) << kRingEBits) | (upper ? static_cast<uint32_t>(kRingUpperBit) : 0u) |
                             (rec ? kRingRecordBit : 0u));
      m.z = static_cast<int>(static_cast<uint32_t>(m.z) | ((lay.bytes >> 4) << kRingOffBits));
      R.meta[static_cast<size_t>(R.tileLevel[T]) + l] = m;
    }
    for (size_t i = 0; i < tr[T].vals.size(); ++i) {
      R.valPos[vOff[T] + i] = static_cast<i32>((off + tr[T].vals[i].first) / vs);
      R.valSrc[vOff[T] + i] = tr[T].vals[i].second;
    }
    for (size_t i = 0; i < tr[T].invs.size(); ++i) {
      R.invPos[iOff[T] + i] = static_cast<i32>((off + tr[T].invs[i].first) / vs);
      R.invSrc[iOff[T] + i] = tr[T].invs[i].second;
    }
  });
  return R;
}

void checkLevelRing(const HostMatrix& H, const HostRing& R, bool dilu, DType vt) {
  const i64 vs = static_cast<i64>(dtypeSize(vt));
  const i64 entSize = vs == 4 ? 8 : 16;
  auto bad = [](i32 G, i64 l, const std::string& what) {
    fail(GR_EINVAL, "level ring check: block " + std::to_string(G) + " level " + std::to_string(l) + ": " + what);
  };
  const i32 group = R.group;
  const bool gs = R.kind != RingKind::Ilu;
  const i32 NG = group > 0 ? (H.P + group - 1) / group : -1;
  if (NG < 1 || static_cast<i32>(R.tileOffset.size()) != NG + 1 || static_cast<i32>(R.tileLevel.size()) != NG + 1 ||
      static_cast<i32>(R.groupStart.size()) != NG + 1)
    fail(GR_EINVAL, "level ring check: table sizes");
  if (gs && (group != 1 || static_cast<i32>(R.haloStart.size()) != H.P + 1 ||
             static_cast<i64>(R.haloSrc.size()) != static_cast<i64>(R.haloStart.back())))
    fail(GR_EINVAL, "level ring check: Gauss-Seidel tables");
  for (i32 G = 0; G < NG; ++G) {
    const i32 T0 = G * group, T1 = std::min<i32>(H.P, T0 + group);
    const i64 gBase = H.tileStart[T0], gRows = H.tileStart[T1] - gBase;
    if (R.groupStart[G] != gBase || R.groupStart[G + 1] != H.tileStart[T1]) bad(G, -1, "block rows");
    std::vector<i32> tileOf(gRows);
    i32 nLower = 0, nUpper = 0;
    for (i32 T = T0; T < T1; ++T) {
      for (i64 p = H.tileStart[T]; p < H.tileStart[T + 1]; ++p) tileOf[p - gBase] = T;
      nLower = std::max(nLower, H.nLowerLevels[T]);
      nUpper = std::max(nUpper, H.nUpperLevels[T]);
    }
    const i64 L = R.tileLevel[G + 1] - R.tileLevel[G];
    if (L != (gs ? nLower : nLower + nUpper)) bad(G, -1, "level count");
    // Gauss-Seidel slots: this sweep's values, the sweep-start values, the
    // halo, the zero slot.
    const i64 nHalo = gs ? H.tiles[T0].nHalo : 0;
    if (gs) {
      for (i64 h = 0; h < nHalo; ++h) {
        const i32 src = R.haloSrc[R.haloStart[T0] + h];
        if (src < 0 || src >= H.n || (src >= gBase && src < gBase + gRows)) bad(G, -1, "halo source");
      }
    }
    std::vector<char> doneL(gRows, 0), doneU(gRows, 0);
    std::vector<i64> inLevel(gRows, -1);  // the level a row is in, once seen
    std::vector<i64> ringOff(L), size(L);
    i64 src = R.tileOffset[G], prevIa = -1;
    for (i64 l = 0; l < L; ++l) {
      const int4 a = R.meta[R.tileLevel[G] + l];
      const i64 k = RingLevelCode::k(a), E = RingLevelCode::E(a), off = RingLevelCode::ringOffset(a);
      const i64 ia = RingLevelCode::issueAfter(a);
      const bool upper = RingLevelCode::upper(a);
      if (upper != (l >= nLower)) bad(G, l, "sweep flag");
      const bool hasInv = gs || upper || dilu;
      const bool rec = RingLevelCode::record(a);
      if (rec && !ringRecordLevel(static_cast<uint32_t>(E), static_cast<uint32_t>(vs), R.compact))
        bad(G, l, "record level");
      const i64 idB = R.compact ? 2 : 4;
      const i64 rowsB = pad16(idB * k), invB = hasInv ? pad16(vs * k) : 0;
      const i64 colsB = R.compact ? pad16(2 * E * k) : pad16(entSize * E * k);
      const i64 valsB = R.compact ? pad16(vs * E * k) : 0;
      const i64 recWord = hasInv ? 8 : 4;
      const i64 S = rec ? 16 * k + pad16(recWord * k) : rowsB + invB + colsB + valsB;
      if (k < 1 || E < 0 || S > R.ringBytes) bad(G, l, "block layout");
      const RingLevelLayout lay = ringLevelLayout(static_cast<uint32_t>(k), static_cast<uint32_t>(E), hasInv,
                                                  static_cast<uint32_t>(vs), R.compact, rec);
      if (rec ? (lay.ents != 16 * k || lay.bytes != S)
              : (lay.inv != rowsB || lay.ents != rowsB + invB || lay.bytes != S ||
                 lay.vals != (R.compact ? rowsB + invB + colsB : rowsB + invB)))
        bad(G, l, "block layout");
      if (RingLevelCode::ents(a) != lay.ents || RingLevelCode::bytes(a) != lay.bytes) bad(G, l, "block layout");
      const i64 entOff = rowsB + invB;
      if (off < 0 || off % 16 != 0 || off + S > R.ringBytes) bad(G, l, "ring offset");
      if (ia < -1 || ia < prevIa || ia < l - kRingBarriers || (l >= 1 && ia > l - 2) || (l == 0 && ia != -1))
        bad(G, l, "copy order");
      ringOff[l] = off;
      size[l] = S;
      // Levels issued before this one and not yet consumed when it is copied.
      for (i64 j = ia + 1; j < l; ++j)
        if (overlaps(ringOff[j], size[j], off, S)) bad(G, l, "copy overwrites level " + std::to_string(j));
      if (src + S > static_cast<i64>(R.bytes.size())) bad(G, l, "source range");
      const uint8_t* blk = R.bytes.data() + src;
      std::vector<char>& done = upper ? doneU : doneL;
      std::vector<i64> rows(k);
      auto rowId = [&](i64 q) {
        i32 il;
        if (rec) {
          uint32_t w2;
          std::memcpy(&w2, blk + lay.ents + recWord * q, 4);
          il = static_cast<i32>(w2 >> 16);
        } else if (R.compact) {
          uint16_t r16;
          std::memcpy(&r16, blk + 2 * q, 2);
          il = r16;
        } else {
          std::memcpy(&il, blk + 4 * q, 4);
        }
        return il;
      };
      for (i64 q = 0; q < k; ++q) {  // the level's rows, for the in-place test
        const i32 il = rowId(q);
        if (il >= 0 && il < gRows) inLevel[il] = l;
      }
      for (i64 q = 0; q < k; ++q) {
        const i32 il = rowId(q);
        uint32_t recW01 = 0, recW2 = 0;
        if (rec) {
          std::memcpy(&recW01, blk + 16 * q + 12, 4);
          std::memcpy(&recW2, blk + lay.ents + recWord * q, 4);
        }
        if (il < 0 || il >= gRows || done[il]) bad(G, l, "row id");
        rows[q] = il;
        for (i64 e = 0; e < E; ++e) {
          i32 c;
          if (rec) {
            c = static_cast<i32>(e == 0 ? (recW01 & 0xFFFFu) : e == 1 ? (recW01 >> 16) : (recW2 & 0xFFFFu));
          } else if (R.compact) {
            uint16_t c16;
            std::memcpy(&c16, blk + entOff + 2 * (e * k + q), 2);
            c = c16;
          } else {
            std::memcpy(&c, blk + entOff + entSize * (e * k + q), 4);
          }
          if (gs) {
            // New value of an earlier row, start value of a later row or of
            // a halo cell, or the zero slot (lower-only rings: no start
            // values). In place, a later row's start value is its own slot,
            // which no row of this or an earlier level may have written.
            const bool lowerOnly = R.kind == RingKind::GaussSeidelLower;
            const i64 haloBase = (R.gsInPlace ? 1 : 2) * gRows;
            if (c < 0 || c > haloBase + nHalo) bad(G, l, "column index");
            if (c < gRows && c < il && !done[c]) bad(G, l, "dependency order");
            if (c < gRows && c >= il) {
              if (!R.gsInPlace || c == il || lowerOnly) bad(G, l, "dependency order");
              if (done[c] || inLevel[c] == l) bad(G, l, "start value overwritten");
            }
            if (!R.gsInPlace && c >= gRows && c < 2 * gRows && (lowerOnly || c - gRows <= il)) bad(G, l, "start value");
            if (c >= haloBase && c < haloBase + nHalo && lowerOnly) bad(G, l, "halo in a lower-only ring");
            continue;
          }
          if (c < 0 || c > gRows) bad(G, l, "column index");
          if (c < gRows && (tileOf[c] != tileOf[il] || !done[c] || (upper ? c <= il : c >= il)))
            bad(G, l, "dependency order");
        }
      }
      for (i64 il : rows) done[il] = 1;
      src += S;
      prevIa = ia;
    }
    if (src != R.tileOffset[G + 1]) bad(G, L, "stream length");
    for (i64 i = 0; i < gRows; ++i)
      if (!doneL[i] || (!gs && !doneU[i])) bad(G, L, "row not covered");
  }
}

LevelRing& DeviceMatrix::levelRing(bool dilu, i64 ringBytes, i32 group, bool allowCompact, RingKind kind,
                                   bool records) {
  auto key = std::make_tuple(dilu, ringBytes, group, allowCompact, static_cast<int>(kind), records);
  auto it = levelRings.find(key);
  if (it != levelRings.end()) return *it->second;
  RingBudget budget;
  budget.numSMs = numSMs;
  int dev = 0, v = 0;
  GR_CUDA(cudaGetDevice(&dev));
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess && v > 0)
    budget.smemPerSM = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess)
    budget.reservedPerBlock = v;
  if (const int b = ringBlocksPerSMWithoutSmem(vt, kind); b > 0) budget.maxBlocksPerSM = b;
  HostRing H = buildLevelRing(*host, dilu, vt, ringBytes, group, budget, allowCompact, kind, records);
  auto R = std::make_unique<LevelRing>();
  R->dilu = dilu;
  R->bytes = static_cast<i64>(H.bytes.size());
  R->ringBytes = H.ringBytes;
  R->maxTileLevels = H.maxTileLevels;
  R->nVal = static_cast<i64>(H.valPos.size());
  R->nInv = static_cast<i64>(H.invPos.size());
  R->tileOffset.upload(H.tileOffset);
  R->templ.upload(H.bytes);
  R->meta.upload(H.meta);
  R->tileLevel.upload(H.tileLevel);
  R->groupStart.upload(H.groupStart);
  R->group = H.group;
  R->compact = H.compact;
  R->numGroups = static_cast<i32>(H.groupStart.size()) - 1;
  R->maxGroupRows = H.maxGroupRows;
  R->valPos.upload(H.valPos);
  R->valSrc.upload(H.valSrc);
  R->invPos.upload(H.invPos);
  R->invSrc.upload(H.invSrc);
  R->kind = H.kind;
  R->maxXSlots = H.maxXSlots;
  R->gsInPlace = H.gsInPlace;
  if (H.kind != RingKind::Ilu) {
    R->haloStart.upload(H.haloStart);
    if (!H.haloSrc.empty()) R->haloSrc.upload(H.haloSrc);
  }
  LevelRing& ref = *R;
  levelRings[key] = std::move(R);
  return ref;
}

}  // namespace gr

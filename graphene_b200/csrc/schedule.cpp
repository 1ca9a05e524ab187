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

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

}  // namespace gr

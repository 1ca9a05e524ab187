// Host-side matrix pipeline of graphene_b200. See host_matrix.hpp.
#include "host_matrix.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>

namespace gr {

bool traceEnabled() {
  static const bool on = [] {
    const char* v = std::getenv("GR_TRACE");
    return v && *v && std::string(v) != "0";
  }();
  return on;
}

TraceScope::TraceScope(const char* name) : name_(name) {
  if (traceEnabled())
    t0_ = std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
              .count();
}

TraceScope::~TraceScope() {
  if (t0_ < 0) return;
  const int64_t t1 =
      std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count();
  std::fprintf(stderr, "[graphene_b200] %s: %.3f ms\n", name_, static_cast<double>(t1 - t0_) * 1e-6);
}

namespace {

double roundTo(DType t, double v) {
  if (t == DType::F32) return static_cast<double>(static_cast<float>(v));
  return v;
}

// Exclusive prefix sum of counts into offsets (size n+1).
std::vector<i64> prefixOffsets(const std::vector<i64>& counts) {
  std::vector<i64> off(counts.size() + 1, 0);
  for (size_t i = 0; i < counts.size(); ++i) off[i + 1] = off[i] + counts[i];
  return off;
}

}  // namespace

// ---------------------------------------------------------------------------
// Construction from triplets: sort by (row, col) and split off the diagonal.
// Reference: sortTripletMatrx (CoordinateFormat.cpp:29-40) followed by
// CRSHostMatrix::convertToCRS (CRSHostMatrix.cpp:88-137). A counting sort by
// row plus a per-row sort by column gives the same order as the reference's
// std::sort on (row, col) for duplicate-free input; duplicates are rejected
// because the reference's downstream steps treat them inconsistently (a
// std::set of columns but a std::set of (column, value) pairs).
std::shared_ptr<HostMatrix> HostMatrix::fromCoo(Coo coo, i64 numTiles, gr_partitioner part,
                                                const i32* rowToTileIn, const double* coords,
                                                DType valueType) {
  if (coo.nrows <= 0) fail(GR_EINVAL, "matrix must have at least one row");
  if (coo.nrows != coo.ncols) fail(GR_EINVAL, "matrix must be square");
  if (coo.row.size() != coo.col.size() || coo.row.size() != coo.val.size())
    fail(GR_EINVAL, "triplet arrays differ in length");
  const i64 n = coo.nrows;
  const i64 nnz = static_cast<i64>(coo.row.size());
  for (i64 i = 0; i < nnz; ++i) {
    if (coo.row[i] < 0 || coo.row[i] >= n || coo.col[i] < 0 || coo.col[i] >= n)
      fail(GR_EINVAL, "triplet index out of range at entry " + std::to_string(i));
  }
  std::vector<i64> counts(n, 0);
  for (i64 i = 0; i < nnz; ++i) counts[coo.row[i]]++;
  std::vector<i64> rowPtr = prefixOffsets(counts);
  std::vector<i64> fill(rowPtr.begin(), rowPtr.end() - 1);
  std::vector<i64> col(nnz);
  std::vector<double> val(nnz);
  for (i64 i = 0; i < nnz; ++i) {
    i64 p = fill[coo.row[i]]++;
    col[p] = coo.col[i];
    val[p] = coo.val[i];
  }
  coo = Coo();  // release
  // Sort each row by column.
  parallelChunks(n, [&](i64 b, i64 e) {
    std::vector<std::pair<i64, double>> tmp;
    for (i64 r = b; r < e; ++r) {
      i64 s = rowPtr[r], t = rowPtr[r + 1];
      bool sorted = true;
      for (i64 k = s + 1; k < t; ++k)
        if (col[k - 1] >= col[k]) { sorted = false; break; }
      if (sorted) continue;
      tmp.clear();
      for (i64 k = s; k < t; ++k) tmp.emplace_back(col[k], val[k]);
      std::sort(tmp.begin(), tmp.end(),
                [](const auto& a, const auto& b) { return a.first < b.first; });
      for (i64 k = s; k < t; ++k) {
        col[k] = tmp[k - s].first;
        val[k] = tmp[k - s].second;
      }
    }
  });
  std::vector<double> crd;
  if (coords) crd.assign(coords, coords + 3 * n);
  return fromSortedCsr(n, std::move(rowPtr), std::move(col), std::move(val), numTiles, part,
                       rowToTileIn, std::move(crd), valueType);
}

std::shared_ptr<HostMatrix> HostMatrix::fromSortedCsr(i64 n, std::vector<i64> rowPtr,
                                                      std::vector<i64> col,
                                                      std::vector<double> val, i64 numTiles,
                                                      gr_partitioner part,
                                                      const i32* rowToTileIn,
                                                      std::vector<double> coords,
                                                      DType valueType) {
  if (valueType == DType::DW)
    fail(GR_EUNSUPPORTED, "twofloat32 matrix coefficients are not supported (use float32 or float64)");
  if (n <= 0) fail(GR_EINVAL, "matrix must have at least one row");
  if (n >= (i64(1) << 31) - 1) fail(GR_EUNSUPPORTED, "more than 2^31-2 rows");
  auto A = std::make_shared<HostMatrix>();
  A->valueType = valueType;
  A->n = n;
  A->coords = std::move(coords);
  {
  GR_TRACE_SCOPE("split diagonal");
  // Split off the diagonal (CRSHostMatrix.cpp:96-132). A missing diagonal
  // stays 0.
  std::vector<i64> offCount(n, 0);
  std::atomic<bool> dup{false};
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e; ++r) {
      i64 c = 0;
      for (i64 k = rowPtr[r]; k < rowPtr[r + 1]; ++k) {
        if (k > rowPtr[r] && col[k - 1] == col[k]) dup = true;
        if (col[k] != r) ++c;
      }
      offCount[r] = c;
    }
  });
  if (dup) fail(GR_EINVAL, "duplicate (row, col) entries are not supported");
  A->gRowPtr = prefixOffsets(offCount);
  A->m = A->gRowPtr[n];
  if (A->m >= (i64(1) << 31) - 1) fail(GR_EUNSUPPORTED, "more than 2^31-2 off-diagonal entries");
  A->gCol.resize(A->m);
  A->gVal.resize(A->m);
  A->gDiag.assign(n, 0.0);
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e; ++r) {
      i64 o = A->gRowPtr[r];
      for (i64 k = rowPtr[r]; k < rowPtr[r + 1]; ++k) {
        if (col[k] == r) {
          A->gDiag[r] = roundTo(valueType, val[k]);
        } else {
          A->gCol[o] = col[k];
          A->gVal[o] = roundTo(valueType, val[k]);
          ++o;
        }
      }
    }
  });
  rowPtr.clear(); rowPtr.shrink_to_fit();
  col.clear(); col.shrink_to_fit();
  val.clear(); val.shrink_to_fit();
  }
  A->buildFromGlobalCrs(numTiles, part, rowToTileIn);
  return A;
}

// ---------------------------------------------------------------------------
// Partitioning and empty-part removal (CRSHostMatrix.cpp:139-271).
void HostMatrix::buildFromGlobalCrs(i64 numTiles, gr_partitioner part, const i32* rowToTileIn) {
  GR_TRACE_SCOPE("host layout (partition, tiles, local CRS, levels)");
  if (numTiles <= 0) fail(GR_EINVAL, "numTiles must be positive");
  if (numTiles > (i64(1) << 30)) fail(GR_EINVAL, "numTiles too large");
  std::vector<i32> raw;
  {
  GR_TRACE_SCOPE("partition");
  if (numTiles == 1 && part != GR_PART_EXPLICIT) {
    // Single tile: no partitioning (CRSHostMatrix.cpp:151-158).
    raw.assign(n, 0);
  } else {
    switch (part) {
      case GR_PART_EXPLICIT:
        if (!rowToTileIn) fail(GR_EINVAL, "explicit partitioning needs row_to_tile");
        raw.assign(rowToTileIn, rowToTileIn + n);
        for (i64 r = 0; r < n; ++r)
          if (raw[r] < 0 || raw[r] >= numTiles)
            fail(GR_EINVAL, "row_to_tile entry out of range at row " + std::to_string(r));
        break;
      case GR_PART_CONTIGUOUS:
        raw = partitionContiguous(*this, static_cast<i32>(numTiles));
        break;
      case GR_PART_RCB:
        if (coords.empty()) fail(GR_EINVAL, "RCB partitioning needs row coordinates");
        raw = partitionRcb(*this, static_cast<i32>(numTiles));
        break;
      case GR_PART_BFS:
        raw = partitionBfs(*this, static_cast<i32>(numTiles));
        break;
      case GR_PART_MULTILEVEL:
        raw = partitionMultilevel(*this, static_cast<i32>(numTiles));
        break;
      case GR_PART_AUTO:
        raw = coords.empty() ? partitionMultilevel(*this, static_cast<i32>(numTiles))
                             : partitionRcb(*this, static_cast<i32>(numTiles));
        break;
      default:
        fail(GR_EINVAL, "unknown partitioner");
    }
  }
  }
  // Remove empty parts, keeping the relative order of the others.
  std::vector<i64> perPart(numTiles, 0);
  for (i64 r = 0; r < n; ++r) perPart[raw[r]]++;
  std::vector<i32> shifted(numTiles, -1);
  i32 next = 0;
  for (i64 t = 0; t < numTiles; ++t)
    if (perPart[t] > 0) shifted[t] = next++;
  P = next;
  rowToTile.resize(n);
  for (i64 r = 0; r < n; ++r) rowToTile[r] = shifted[raw[r]];
  buildTileLayout();
  buildLocalCrs();
  buildLevels();
  computeStructureKey();
}

// splitmix64-style mixing of the pattern, in parallel chunks combined in
// order (the key does not depend on the thread count).
void HostMatrix::computeStructureKey() {
  auto mix = [](u64 h, u64 v) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
    return h ^ (h >> 27);
  };
  const i64 chunk = i64(1) << 16;
  const i64 nc = (std::max(n, m) + chunk - 1) / chunk;
  std::vector<u64> part(static_cast<size_t>(nc) + 1, 0);
  parallelFor(nc, [&](i64 c) {
    u64 h = static_cast<u64>(c);
    for (i64 i = c * chunk; i < std::min(m, (c + 1) * chunk); ++i) h = mix(h, static_cast<u64>(gCol[i]));
    for (i64 i = c * chunk; i < std::min(n, (c + 1) * chunk); ++i)
      h = mix(mix(h, static_cast<u64>(gRowPtr[i + 1])), static_cast<u64>(rowToTile[i]));
    part[c] = h;
  });
  u64 h = mix(mix(mix(static_cast<u64>(n), static_cast<u64>(m)), static_cast<u64>(P)),
              static_cast<u64>(valueType) * 16 + static_cast<u64>(format));
  for (i64 c = 0; c < nc; ++c) h = mix(h, part[c]);
  structureKey = h == 0 ? 1 : h;
}

void HostMatrix::localValues(const double* gv, const double* gd, std::vector<double>& off,
                             std::vector<double>& dg) const {
  if (static_cast<i64>(localSrc.size()) != m) fail(GR_EUNSUPPORTED, "no tile-local entry map");
  off.resize(m);
  dg.resize(n);
  parallelChunks(m, [&](i64 b, i64 e) {
    for (i64 p = b; p < e; ++p) off[p] = roundTo(valueType, gv[localSrc[p]]);
  });
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 p = b; p < e; ++p) dg[p] = roundTo(valueType, gd[iperm[p]]);
  });
}

std::shared_ptr<HostMatrix> HostMatrix::withGlobalValues(const HostMatrix& like, const double* gv,
                                                         const double* gd) {
  if (like.format != GR_FORMAT_CRS || !like.sumRank.empty())
    fail(GR_EUNSUPPORTED, "values-only updates are for CRS matrices");
  auto A = std::make_shared<HostMatrix>(like);
  parallelChunks(like.m, [&](i64 b, i64 e) {
    for (i64 k = b; k < e; ++k) A->gVal[k] = roundTo(like.valueType, gv[k]);
  });
  parallelChunks(like.n, [&](i64 b, i64 e) {
    for (i64 k = b; k < e; ++k) A->gDiag[k] = roundTo(like.valueType, gd[k]);
  });
  like.localValues(gv, gd, A->offDiag, A->diag);
  return A;
}

std::shared_ptr<HostMatrix> HostMatrix::withValues(const HostMatrix& like, const std::vector<i64>& rowPtr,
                                                   const std::vector<i64>& col, const std::vector<double>& val) {
  if (like.format != GR_FORMAT_CRS || !like.sumRank.empty())
    fail(GR_EUNSUPPORTED, "values-only updates are for CRS matrices");
  if (static_cast<i64>(rowPtr.size()) != like.n + 1 || static_cast<i64>(col.size()) != like.n + like.m ||
      col.size() != val.size() || static_cast<i64>(like.localSrc.size()) != like.m)
    fail(GR_EINVAL, "the new values do not have the template matrix's pattern");
  GR_TRACE_SCOPE("values on a template's structure");
  auto A = std::make_shared<HostMatrix>(like);
  std::atomic<bool> bad{false};
  parallelChunks(like.n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e && !bad; ++r) {
      i64 o = like.gRowPtr[r];
      bool diagSeen = false;
      for (i64 k = rowPtr[r]; k < rowPtr[r + 1]; ++k) {
        if (col[k] == r) {
          A->gDiag[r] = roundTo(like.valueType, val[k]);
          diagSeen = true;
        } else {
          if (o >= like.gRowPtr[r + 1] || like.gCol[o] != col[k]) {
            bad = true;
            break;
          }
          A->gVal[o++] = roundTo(like.valueType, val[k]);
        }
      }
      if (o != like.gRowPtr[r + 1] || !diagSeen) bad = true;
    }
  });
  if (bad) fail(GR_EINVAL, "the new values do not have the template matrix's pattern");
  parallelChunks(like.m, [&](i64 b, i64 e) {
    for (i64 p = b; p < e; ++p) A->offDiag[p] = A->gVal[like.localSrc[p]];
  });
  parallelChunks(like.n, [&](i64 b, i64 e) {
    for (i64 p = b; p < e; ++p) A->diag[p] = A->gDiag[like.iperm[p]];
  });
  return A;
}

// ---------------------------------------------------------------------------
// Tile layout (CRSHostMatrix.cpp:273-354, DistributedTileLayout.cpp:63-126).
// A row is a separator row when one of its columns lives on another tile;
// separator rows are grouped into regions keyed by the set of those tiles,
// regions numbered in order of first appearance in an ascending row scan.
// The halo regions of a tile are ordered by (source tile, creation order of
// the source's region): the order the reference produces when its parallel
// loop over tiles runs sequentially (the reference's own order depends on
// thread timing).
void HostMatrix::buildTileLayout() {
  GR_TRACE_SCOPE("tile layout");
  // Rows of each tile in ascending order.
  std::vector<i64> cnt(P, 0);
  for (i64 r = 0; r < n; ++r) cnt[rowToTile[r]]++;
  std::vector<i64> start = prefixOffsets(cnt);
  std::vector<i64> rowsByTile(n);
  {
    std::vector<i64> f(start.begin(), start.end() - 1);
    for (i64 r = 0; r < n; ++r) rowsByTile[f[rowToTile[r]]++] = r;
  }
  struct LocalRegion {
    std::vector<i32> dst;
    std::vector<i64> cells;
  };
  std::vector<std::vector<LocalRegion>> local(P);
  tiles.assign(P, Tile());
  parallelFor(P, [&](i64 T) {
    std::map<std::vector<i32>, i32> index;
    std::vector<i32> nb;
    auto& tile = tiles[T];
    auto& regs = local[T];
    for (i64 q = start[T]; q < start[T + 1]; ++q) {
      i64 r = rowsByTile[q];
      nb.clear();
      for (i64 k = gRowPtr[r]; k < gRowPtr[r + 1]; ++k) {
        i32 t = rowToTile[gCol[k]];
        if (t != T) nb.push_back(t);
      }
      if (nb.empty()) {
        tile.interior.push_back(r);
        continue;
      }
      std::sort(nb.begin(), nb.end());
      nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
      auto it = index.find(nb);
      i32 id;
      if (it == index.end()) {
        id = static_cast<i32>(regs.size());
        index.emplace(nb, id);
        regs.push_back(LocalRegion{nb, {}});
      } else {
        id = it->second;
      }
      regs[id].cells.push_back(r);
    }
    tile.nInterior = static_cast<i64>(tile.interior.size());
  });
  regions.clear();
  for (i32 T = 0; T < P; ++T) {
    for (auto& lr : local[T]) {
      tiles[T].sepRegions.push_back(static_cast<i32>(regions.size()));
      tiles[T].nSeparator += static_cast<i64>(lr.cells.size());
      regions.push_back(Region{T, std::move(lr.dst), std::move(lr.cells)});
    }
  }
  local.clear();
  regionOf.assign(n, -1);
  idxInRegion.assign(n, 0);
  parallelFor(static_cast<i64>(regions.size()), [&](i64 R) {
    const auto& reg = regions[R];
    for (size_t i = 0; i < reg.cells.size(); ++i) {
      regionOf[reg.cells[i]] = static_cast<i32>(R);
      idxInRegion[reg.cells[i]] = static_cast<i32>(i);
    }
  });
  for (i32 S = 0; S < P; ++S)
    for (i32 R : tiles[S].sepRegions)
      for (i32 T : regions[R].dst) tiles[T].haloRegions.push_back(R);
  numHaloTotal = 0;
  maxTileRows = 0;
  for (i32 T = 0; T < P; ++T) {
    auto& tile = tiles[T];
    i64 off = tile.rows();
    tile.haloOffset.clear();
    for (i32 R : tile.haloRegions) {
      tile.haloOffset.emplace_back(R, off);
      off += static_cast<i64>(regions[R].cells.size());
    }
    tile.nHalo = off - tile.rows();
    std::sort(tile.haloOffset.begin(), tile.haloOffset.end());
    numHaloTotal += tile.nHalo;
    maxTileRows = std::max(maxTileRows, tile.rows());
  }
  tileStart.assign(P + 1, 0);
  for (i32 T = 0; T < P; ++T) tileStart[T + 1] = tileStart[T] + tiles[T].rows();
  perm.assign(n, 0);
  iperm.assign(n, 0);
  parallelFor(P, [&](i64 T) {
    const auto& tile = tiles[T];
    i64 p = tileStart[T];
    for (i64 r : tile.interior) { perm[r] = static_cast<i32>(p); iperm[p] = static_cast<i32>(r); ++p; }
    for (i32 R : tile.sepRegions)
      for (i64 r : regions[R].cells) { perm[r] = static_cast<i32>(p); iperm[p] = static_cast<i32>(r); ++p; }
  });
}

// ---------------------------------------------------------------------------
// Tile-local CRS (CRSHostMatrix.cpp:379-432 for the columns, :466-525 for the
// values): each row's columns translated to tile-local ids and sorted by
// them, so interior columns come first, then separator, then halo columns.
void HostMatrix::buildLocalCrs() {
  GR_TRACE_SCOPE("tile-local CRS");
  rowPtr.assign(n + 1, 0);
  for (i64 p = 0; p < n; ++p) {
    i64 g = iperm[p];
    rowPtr[p + 1] = rowPtr[p] + (gRowPtr[g + 1] - gRowPtr[g]);
  }
  colPerm.assign(m, 0);
  colLocal.assign(m, 0);
  offDiag.assign(m, 0.0);
  localSrc.assign(m, 0);
  diag.assign(n, 0.0);
  parallelFor(P, [&](i64 T) {
    const auto& tile = tiles[T];
    const i64 base = tileStart[T];
    const i64 nRows = tile.rows();
    std::vector<std::pair<i64, i64>> ent;  // (local column, global entry)
    for (i64 p = base; p < base + nRows; ++p) {
      i64 g = iperm[p];
      diag[p] = gDiag[g];
      ent.clear();
      for (i64 k = gRowPtr[g]; k < gRowPtr[g + 1]; ++k) {
        i64 c = gCol[k];
        i64 lc;
        if (rowToTile[c] == T) {
          lc = perm[c] - base;
        } else {
          // The halo of T holds only rows of other tiles that reference T
          // themselves; a one-sided coupling has no halo cell, which makes
          // the reference's globalToLocalRow.at() throw
          // (CRSHostMatrix.cpp:415).
          i32 R = regionOf[c];
          auto it = std::lower_bound(tile.haloOffset.begin(), tile.haloOffset.end(),
                                     std::make_pair(R, i64(-1)));
          if (R < 0 || it == tile.haloOffset.end() || it->first != R)
            fail(GR_EUNSUPPORTED,
                 "matrix structure is not symmetric across tiles: row " + std::to_string(g) +
                     " references row " + std::to_string(c) + " of another tile, which does not "
                     "reference back");
          lc = it->second + idxInRegion[c];
        }
        ent.emplace_back(lc, k);
      }
      std::sort(ent.begin(), ent.end());
      i64 o = rowPtr[p];
      for (auto& [lc, k] : ent) {
        colLocal[o] = static_cast<i32>(lc);
        colPerm[o] = perm[gCol[k]];
        offDiag[o] = gVal[k];
        localSrc[o] = static_cast<i32>(k);
        ++o;
      }
    }
  });
}

// ---------------------------------------------------------------------------
// Level sets per tile. The lower level of a row is one more than the largest
// lower level among its lower-triangular tile-local neighbours (0 if none);
// this is the colour the reference's wave algorithm assigns
// (CRSHostMatrix.cpp:527-614) for structurally symmetric tiles, and stays a
// valid schedule for unsymmetric ones. Upper levels are the same for the
// upper-triangular DAG, used by the backward sweep.
void HostMatrix::buildLevels() {
  GR_TRACE_SCOPE("level sets");
  lowerLevel.assign(n, 0);
  upperLevel.assign(n, 0);
  nLowerLevels.assign(P, 0);
  nUpperLevels.assign(P, 0);
  parallelFor(P, [&](i64 T) {
    const i64 base = tileStart[T];
    const i64 nRows = tiles[T].rows();
    i32 maxL = -1, maxU = -1;
    for (i64 i = 0; i < nRows; ++i) {
      i64 p = base + i;
      i32 lv = 0;
      for (i64 k = rowPtr[p]; k < rowPtr[p + 1]; ++k) {
        i64 c = colLocal[k];
        if (c >= i) break;
        lv = std::max(lv, lowerLevel[base + c] + 1);
      }
      lowerLevel[p] = lv;
      maxL = std::max(maxL, lv);
    }
    for (i64 i = nRows - 1; i >= 0; --i) {
      i64 p = base + i;
      i32 lv = 0;
      for (i64 k = rowPtr[p + 1] - 1; k >= rowPtr[p]; --k) {
        i64 c = colLocal[k];
        if (c < i) break;
        if (c >= nRows) continue;
        lv = std::max(lv, upperLevel[base + c] + 1);
      }
      upperLevel[p] = lv;
      maxU = std::max(maxU, lv);
    }
    nLowerLevels[T] = maxL + 1;
    nUpperLevels[T] = maxU + 1;
  });
  // "Multicolour recommended" when more than 90 % of the rows sit in colours
  // holding more than 12 rows (CRSHostMatrix.cpp:648-669).
  i64 parallelRows = 0;
  for (i32 T = 0; T < P; ++T) {
    std::vector<i64> sz(nLowerLevels[T], 0);
    for (i64 p = tileStart[T]; p < tileStart[T + 1]; ++p) sz[lowerLevel[p]]++;
    for (i64 s : sz)
      if (s > 12) parallelRows += s;
  }
  multicolorRecommended = static_cast<double>(parallelRows) > 0.9 * static_cast<double>(n);
}

gr_matrix_info HostMatrix::info() const {
  gr_matrix_info i{};
  i.num_rows = n;
  i.num_off_diag = m;
  i.num_tiles = P;
  i.num_halo_total = numHaloTotal;
  i.max_tile_rows = maxTileRows;
  i64 nl = 0, nu = 0;
  for (i32 T = 0; T < P; ++T) { nl += nLowerLevels[T]; nu += nUpperLevels[T]; }
  i.num_lower_levels_total = nl;
  i.num_upper_levels_total = nu;
  i.value_type = static_cast<int32_t>(valueType);
  i.format = format;
  i.multicolor_recommended = multicolorRecommended ? 1 : 0;
  return i;
}

// ---------------------------------------------------------------------------
// Partitioners. All balance the reference's vertex weight (row off-diagonal
// count + 1, CRSHostMatrix.cpp:185-194).
namespace {

inline i64 vertexWeight(const HostMatrix& A, i64 r) { return A.gRowPtr[r + 1] - A.gRowPtr[r] + 1; }

// Index s in [0, cnt] of the weighted split: the smallest prefix whose
// weight reaches total * p1 / parts.
template <class W>
i64 weightedSplit(i64 cnt, i32 p1, i32 parts, W w) {
  i64 total = 0;
  for (i64 i = 0; i < cnt; ++i) total += w(i);
  i64 acc = 0;
  for (i64 i = 0; i < cnt; ++i) {
    if (acc * parts >= total * p1) return i;
    acc += w(i);
  }
  return cnt;
}

}  // namespace

std::vector<i32> partitionContiguous(const HostMatrix& A, i32 numParts) {
  std::vector<i32> part(A.n);
  i64 total = A.m + A.n;
  i64 acc = 0;
  for (i64 r = 0; r < A.n; ++r) {
    i64 p = (acc * numParts) / total;
    part[r] = static_cast<i32>(std::min<i64>(p, numParts - 1));
    acc += vertexWeight(A, r);
  }
  return part;
}

namespace {

// Sorts v ascending by `less`: chunks sorted on the host threads, then
// merged pairwise in parallel rounds. `less` must be a strict total order,
// so that the result equals a sequential sort's.
template <class T, class Less>
void parallelSort(std::vector<T>& v, i64 b, i64 e, Less less) {
  const i64 n = e - b;
  int P = 1;
  while (P * 2 <= hostThreads() && P < 64) P *= 2;
  if (n < (i64(1) << 17) || P == 1) {
    std::sort(v.begin() + b, v.begin() + e, less);
    return;
  }
  std::vector<i64> cut(P + 1);
  for (int t = 0; t <= P; ++t) cut[t] = b + n * t / P;
  parallelFor(P, [&](i64 t) { std::sort(v.begin() + cut[t], v.begin() + cut[t + 1], less); });
  std::vector<T> tmp(static_cast<size_t>(n));
  for (int width = 1; width < P; width *= 2) {
    parallelFor(P / (2 * width), [&](i64 j) {
      const i64 lo = cut[2 * width * j], mid = cut[2 * width * j + width], hi = cut[2 * width * (j + 1)];
      std::merge(v.begin() + lo, v.begin() + mid, v.begin() + mid, v.begin() + hi, tmp.begin() + (lo - b), less);
    });
    std::copy(tmp.begin(), tmp.end(), v.begin() + b);
  }
}

void rcbRec(const HostMatrix& A, i64* rows, i64 cnt, i32 parts, i32 first, i32* out, int depth) {
  if (parts == 1) {
    for (i64 i = 0; i < cnt; ++i) out[rows[i]] = first;
    return;
  }
  if (cnt == 0) return;
  const double* c = A.coords.data();
  double lo[3] = {c[3 * rows[0]], c[3 * rows[0] + 1], c[3 * rows[0] + 2]};
  double hi[3] = {lo[0], lo[1], lo[2]};
  for (i64 i = 1; i < cnt; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], c[3 * rows[i] + d]);
      hi[d] = std::max(hi[d], c[3 * rows[i] + d]);
    }
  int axis = 0;
  for (int d = 1; d < 3; ++d)
    if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
  // Rows by (coordinate along the axis, row), sorted as contiguous
  // (key, row) pairs.
  {
    std::vector<std::pair<double, i64>> kv(cnt);
    for (i64 i = 0; i < cnt; ++i) kv[i] = {c[3 * rows[i] + axis], rows[i]};
    parallelSort(kv, 0, cnt, std::less<std::pair<double, i64>>());
    for (i64 i = 0; i < cnt; ++i) rows[i] = kv[i].second;
  }
  i32 p1 = parts / 2;
  auto w = [&](i64 i) { return vertexWeight(A, rows[i]); };
  i64 s = weightedSplit(cnt, p1, parts, w);
  // Snap the cut to the nearest coordinate plane so that regular grids are
  // cut into boxes.
  auto boundary = [&](i64 i) {
    return i == 0 || i == cnt || c[3 * rows[i - 1] + axis] != c[3 * rows[i] + axis];
  };
  if (!boundary(s)) {
    i64 l = s, r = s;
    while (!boundary(l)) --l;
    while (!boundary(r)) ++r;
    i64 total = 0, wl = 0, wr = 0;
    for (i64 i = 0; i < cnt; ++i) {
      total += w(i);
      if (i < l) wl += w(i);
      if (i < r) wr += w(i);
    }
    double target = static_cast<double>(total) * p1 / parts;
    i64 pick = (std::abs(wl - target) <= std::abs(wr - target)) ? l : r;
    if (pick > 0 && pick < cnt) s = pick;
  }
  if (depth < 6 && cnt > 200000) {
    std::thread th([&]() { rcbRec(A, rows, s, p1, first, out, depth + 1); });
    rcbRec(A, rows + s, cnt - s, parts - p1, first + p1, out, depth + 1);
    th.join();
  } else {
    rcbRec(A, rows, s, p1, first, out, depth + 1);
    rcbRec(A, rows + s, cnt - s, parts - p1, first + p1, out, depth + 1);
  }
}

}  // namespace

std::vector<i32> partitionRcb(const HostMatrix& A, i32 numParts) {
  std::vector<i64> rows(A.n);
  std::iota(rows.begin(), rows.end(), 0);
  std::vector<i32> part(A.n, 0);
  rcbRec(A, rows.data(), A.n, numParts, 0, part.data(), 0);
  return part;
}

namespace {

struct BfsState {
  const HostMatrix& A;
  std::vector<i32> label;  // subset label of each row
  std::vector<i32> stamp;  // BFS visit stamp of each row
  std::atomic<i32> nextLabel{1};
  std::atomic<i32> nextStamp{1};
  explicit BfsState(const HostMatrix& a) : A(a), label(a.n, 0), stamp(a.n, 0) {}
};

// BFS over the subset with label lab from v; when the component is
// exhausted, continues from the smallest unvisited subset row, so that the
// returned order covers the whole subset.
void bfsOrder(BfsState& S, const std::vector<i64>& rows, i32 lab, i64 v, std::vector<i64>& order) {
  i32 st = S.nextStamp.fetch_add(1);
  order.clear();
  order.reserve(rows.size());
  size_t head = 0, scan = 0;
  auto visit = [&](i64 r) {
    S.stamp[r] = st;
    order.push_back(r);
  };
  visit(v);
  while (order.size() < rows.size()) {
    if (head == order.size()) {
      while (S.stamp[rows[scan]] == st) ++scan;
      visit(rows[scan]);
    }
    i64 r = order[head++];
    for (i64 k = S.A.gRowPtr[r]; k < S.A.gRowPtr[r + 1]; ++k) {
      i64 c = S.A.gCol[k];
      if (S.label[c] == lab && S.stamp[c] != st) visit(c);
    }
  }
}

void bfsRec(BfsState& S, std::vector<i64> rows, i32 parts, i32 first, i32* out, int depth) {
  if (parts == 1) {
    for (i64 r : rows) out[r] = first;
    return;
  }
  if (rows.empty()) return;
  i32 lab = S.nextLabel.fetch_add(1);
  for (i64 r : rows) S.label[r] = lab;
  std::vector<i64> order;
  i64 v = rows[0];
  for (int it = 0; it < 2; ++it) {
    bfsOrder(S, rows, lab, v, order);
    v = order.back();
  }
  bfsOrder(S, rows, lab, v, order);
  i32 p1 = parts / 2;
  i64 cnt = static_cast<i64>(order.size());
  i64 s = weightedSplit(cnt, p1, parts, [&](i64 i) { return vertexWeight(S.A, order[i]); });
  std::vector<i64> a(order.begin(), order.begin() + s), b(order.begin() + s, order.end());
  std::sort(a.begin(), a.end());
  std::sort(b.begin(), b.end());
  rows.clear();
  rows.shrink_to_fit();
  if (depth < 6 && cnt > 200000) {
    std::thread th([&]() { bfsRec(S, std::move(a), p1, first, out, depth + 1); });
    bfsRec(S, std::move(b), parts - p1, first + p1, out, depth + 1);
    th.join();
  } else {
    bfsRec(S, std::move(a), p1, first, out, depth + 1);
    bfsRec(S, std::move(b), parts - p1, first + p1, out, depth + 1);
  }
}

}  // namespace

std::vector<i32> partitionBfs(const HostMatrix& A, i32 numParts) {
  BfsState S(A);
  std::vector<i64> rows(A.n);
  std::iota(rows.begin(), rows.end(), 0);
  std::vector<i32> part(A.n, 0);
  bfsRec(S, std::move(rows), numParts, 0, part.data(), 0);
  return part;
}

// ---------------------------------------------------------------------------
// 7-point Poisson matrix (matrix/host/details/Poisson.cpp:26-69): diagonal 6,
// off-diagonals -1, row = k*nx*ny + j*nx + i, neighbours outside the grid
// dropped. Rows are emitted sorted by column.
GeneratedCsr generatePoisson(i64 nx, i64 ny, i64 nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) fail(GR_EINVAL, "grid dimensions must be positive");
  GeneratedCsr g;
  g.n = nx * ny * nz;
  const i64 n = g.n;
  g.rowPtr.assign(n + 1, 0);
  auto count = [&](i64 i, i64 j, i64 k) {
    return 1 + (k > 0) + (j > 0) + (i > 0) + (i < nx - 1) + (j < ny - 1) + (k < nz - 1);
  };
  for (i64 r = 0; r < n; ++r) {
    i64 i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
    g.rowPtr[r + 1] = g.rowPtr[r] + count(i, j, k);
  }
  g.col.resize(g.rowPtr[n]);
  g.val.resize(g.rowPtr[n]);
  g.coords.resize(3 * n);
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e; ++r) {
      i64 i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
      i64 o = g.rowPtr[r];
      auto put = [&](i64 c, double v) { g.col[o] = c; g.val[o] = v; ++o; };
      if (k > 0) put(r - nx * ny, -1.0);
      if (j > 0) put(r - nx, -1.0);
      if (i > 0) put(r - 1, -1.0);
      put(r, 6.0);
      if (i < nx - 1) put(r + 1, -1.0);
      if (j < ny - 1) put(r + nx, -1.0);
      if (k < nz - 1) put(r + nx * ny, -1.0);
      g.coords[3 * r] = static_cast<double>(i);
      g.coords[3 * r + 1] = static_cast<double>(j);
      g.coords[3 * r + 2] = static_cast<double>(k);
    }
  });
  return g;
}

}  // namespace gr

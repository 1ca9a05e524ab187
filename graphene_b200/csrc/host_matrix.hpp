// Host-side matrix pipeline: triplets -> CRS with split diagonal -> row
// partition -> interior/separator/halo tile layout -> tile-local CRS ->
// level sets. Follows matrix/host/details/crs/CRSHostMatrix.cpp and
// matrix/host/DistributedTileLayout.cpp of the reference, re-designed for a
// GPU: tiles are stored contiguously in "tile order" (the reference's
// decomposed vector layout), so a tile-local column id maps to a global
// vector index and halo cells need no storage.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.hpp"

namespace gr {

// A matrix in triplet format (matrix/host/details/CoordinateFormat.hpp:29-38).
struct Coo {
  i64 nrows = 0, ncols = 0;
  std::vector<i64> row, col;
  std::vector<double> val;
};

struct HostMatrix {
  DType valueType = DType::F32;
  i64 n = 0;  // rows
  i64 m = 0;  // stored off-diagonal entries
  i32 P = 0;  // tiles after empty-tile removal

  // Global CRS with the diagonal split off (CRSHostMatrix.cpp:88-137).
  std::vector<i64> gRowPtr;
  std::vector<i64> gCol;
  std::vector<double> gVal;   // rounded to valueType
  std::vector<double> gDiag;  // rounded to valueType, 0 when absent
  std::vector<double> coords; // optional, 3 per row (generated grids)

  // Partitioning::rowToTile after empty-tile removal.
  std::vector<i32> rowToTile;

  // A separator region: the rows of one tile that are needed by exactly the
  // tiles in dst (DistributedTileLayout.hpp:269-282).
  struct Region {
    i32 tile = 0;
    std::vector<i32> dst;  // ascending
    std::vector<i64> cells;  // global rows, ascending
  };
  std::vector<Region> regions;  // numbered by (owning tile, creation order)

  struct Tile {
    i64 nInterior = 0, nSeparator = 0, nHalo = 0;
    std::vector<i64> interior;       // global rows, ascending
    std::vector<i32> sepRegions;     // region ids in creation order
    std::vector<i32> haloRegions;    // region ids in canonical order
    std::vector<std::pair<i32, i64>> haloOffset;  // (region id, local offset), sorted by id
    i64 rows() const { return nInterior + nSeparator; }
  };
  std::vector<Tile> tiles;
  std::vector<i64> tileStart;  // P + 1 offsets into tile order
  std::vector<i32> perm;       // global row -> tile-order index
  std::vector<i32> iperm;      // tile-order index -> global row
  std::vector<i32> regionOf;   // global row -> region id (-1 for interior rows)
  std::vector<i32> idxInRegion;

  // Tile-local CRS in tile order: rows are tile-order indices, each row's
  // entries sorted by tile-local column id (CRSHostMatrix.cpp:379-432).
  std::vector<i64> rowPtr;     // n + 1
  std::vector<i32> colPerm;    // column as tile-order index
  std::vector<i32> colLocal;   // tile-local column id (halo ids >= tile rows)
  std::vector<double> offDiag; // values in local order
  std::vector<double> diag;    // tile order

  // Level ("colour") of each row in its tile's lower / upper dependency DAG.
  std::vector<i32> lowerLevel, upperLevel;  // tile order
  std::vector<i32> nLowerLevels, nUpperLevels;  // per tile
  bool multicolorRecommended = false;

  i64 numHaloTotal = 0;
  i64 maxTileRows = 0;

  // Structure identity: a hash of the value type, the sparsity pattern and
  // the tile map. Matrices with equal keys have the same partition, tile
  // layout, tile-local CRS pattern and level sets, so a device copy of one
  // can take the other's values without any host-side layout work.
  u64 structureKey = 0;
  // SpMV column encoding of device copies (SellMatrix): -1 automatic, 0 the
  // 32-bit layout, 1 the 16-bit layout.
  int spmvLayout = -1;
  // Global CRS entry (gVal index) of every tile-local CRS entry.
  std::vector<i32> localSrc;

  // LDU format (matrix/details/ldu/LDUMatrix.cpp:42-168,
  // LDUAddressing.hpp:42-91). The faces in natural numbering, owner <
  // neighbour, sorted by owner; coefficients in face order, rounded to the
  // value type. sumRank gives, for every tile-local CRS entry, its position
  // in its row's LDU summation order (owned faces in face order, then the
  // faces the row neighbours in losort order). All empty for CRS matrices.
  int format = GR_FORMAT_CRS;
  std::vector<i64> lduOwner, lduNeighbour;
  std::vector<double> lduLower, lduUpper, lduDiag;
  std::vector<i32> sumRank;

  // Builds everything from triplets. rowToTileIn is used for
  // GR_PART_EXPLICIT; coords (3 per row) for GR_PART_RCB.
  static std::shared_ptr<HostMatrix> fromCoo(Coo coo, i64 numTiles, gr_partitioner part,
                                             const i32* rowToTileIn, const double* coords,
                                             DType valueType);
  // Same, from a CRS whose rows are already sorted by column (fast path of
  // the generators; identical result to fromCoo on the same entries).
  static std::shared_ptr<HostMatrix> fromSortedCsr(i64 n, std::vector<i64> rowPtr,
                                                   std::vector<i64> col, std::vector<double> val,
                                                   i64 numTiles, gr_partitioner part,
                                                   const i32* rowToTileIn,
                                                   std::vector<double> coords, DType valueType);

  // From LDU arrays: num_faces faces (owner, neighbour, lower, upper) and
  // the diagonal, natural numbering. upper == nullptr means upper = lower.
  static std::shared_ptr<HostMatrix> fromLdu(i64 n, i64 numFaces, const i64* owner, const i64* neighbour,
                                             const double* diag, const double* lower, const double* upper,
                                             i64 numTiles, gr_partitioner part, const i32* rowToTileIn,
                                             const double* coords, DType valueType);

  // The structure of `like` (a CRS matrix) with new values: a natural-order
  // CRS, diagonal included, rows sorted by column, whose pattern must be
  // like's exactly (GR_EINVAL otherwise). Partition, layout and levels are
  // copied, not rebuilt.
  static std::shared_ptr<HostMatrix> withValues(const HostMatrix& like, const std::vector<i64>& rowPtr,
                                                const std::vector<i64>& col, const std::vector<double>& val);

  // Global CRS values of this structure (gVal order, rounded to the value
  // type) converted to the tile-local CRS order and the tile-ordered
  // diagonal, the layout a device matrix takes them in.
  void localValues(const double* gVal, const double* gDiag, std::vector<double>& off,
                   std::vector<double>& dg) const;
  // `like`'s structure with global CRS values (gVal order) and a diagonal.
  static std::shared_ptr<HostMatrix> withGlobalValues(const HostMatrix& like, const double* gVal,
                                                      const double* gDiag);

  gr_matrix_info info() const;

  template <class T>
  void decompose(const T* natural, T* tileOrdered) const {
    parallelChunks(n, [&](i64 b, i64 e) {
      for (i64 p = b; p < e; ++p) tileOrdered[p] = natural[iperm[p]];
    });
  }
  template <class T>
  void compose(const T* tileOrdered, T* natural) const {
    parallelChunks(n, [&](i64 b, i64 e) {
      for (i64 p = b; p < e; ++p) natural[iperm[p]] = tileOrdered[p];
    });
  }

 private:
  void buildFromGlobalCrs(i64 numTiles, gr_partitioner part, const i32* rowToTileIn);
  void buildTileLayout();
  void buildLocalCrs();
  void buildLevels();
  void computeStructureKey();
};

// Row partitioners (raw part ids in [0, numParts), before empty-part removal).
std::vector<i32> partitionContiguous(const HostMatrix& A, i32 numParts);
std::vector<i32> partitionRcb(const HostMatrix& A, i32 numParts);
std::vector<i32> partitionBfs(const HostMatrix& A, i32 numParts);
// Multilevel recursive bisection (partition.cpp): heavy-edge coarsening,
// greedy growing, Fiduccia-Mattheyses refinement; weight = row entries + 1.
std::vector<i32> partitionMultilevel(const HostMatrix& A, i32 numParts);
// Off-diagonal entries whose column lies in another part than their row.
i64 edgeCut(const HostMatrix& A, const std::vector<i32>& rowToTile);

// Generators (rows sorted by column).
struct GeneratedCsr {
  i64 n = 0;
  std::vector<i64> rowPtr, col;
  std::vector<double> val;
  std::vector<double> coords;
};
GeneratedCsr generatePoisson(i64 nx, i64 ny, i64 nz);
GeneratedCsr generateVarPoisson(i64 nx, i64 ny, i64 nz, double sigma, uint64_t seed);
GeneratedCsr generateConvDiff(i64 nx, i64 ny, i64 nz, double vx, double vy, double vz);
void generateUniform(uint64_t seed, i64 n, double lo, double hi, double* out);
// The values of generator `kind` (0 Poisson, 1 variable-coefficient, 2
// convection-diffusion) in a generated matrix's global CRS order: the
// off-diagonals at gVal (gRowPtr offsets), the diagonal at gDiag. The same
// numbers as the full generator; false when gRowPtr is not the grid's.
bool generateValues(int kind, i64 nx, i64 ny, i64 nz, const double* params, uint64_t seed,
                    const std::vector<i64>& gRowPtr, double* gVal, double* gDiag);

// Unstructured-mesh stand-in in LDU form: an nx x ny x nz hexahedral mesh
// with node positions jittered by U(-0.2, 0.2) spacings (jitterSeed; only the
// cell centroids in `coords` depend on it), cell ids permuted (permSeed),
// face owner = smaller cell id, neighbour = larger, faces sorted by (owner,
// neighbour), face coefficient c = 10^U(-2, 2) (coefSeed), off-diagonals -c
// and diagonal = sum of the cell's face coefficients + 1e-3.
struct LduMesh {
  i64 n = 0;
  std::vector<i64> owner, neighbour;
  std::vector<double> lower, upper, diag, coords;
};
LduMesh generateLduMesh(i64 nx, i64 ny, i64 nz, uint64_t jitterSeed, uint64_t permSeed, uint64_t coefSeed);
void generateNormal(uint64_t seed, i64 n, double* out);

// MatrixMarket reader (public format spec; replaces fast_matrix_market).
// Values are parsed directly into valueType (strtof for float32) so that
// they are rounded once, as a reader templated on the value type does.
Coo readMatrixMarket(const std::string& path, DType valueType);
// A vector from a MatrixMarket file (matrix/host/details/MatrixMarket.cpp:66-102):
// a "vector" object (coordinate: index value pairs; array: one value a line)
// or the first column of a "matrix" object (coordinate or array). Entries
// the file does not list are 0; a later entry for an index replaces an
// earlier one. Returns the rows, values rounded once to valueType.
std::vector<double> readMatrixMarketVector(const std::string& path, DType valueType);

}  // namespace gr

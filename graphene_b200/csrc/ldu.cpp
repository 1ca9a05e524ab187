// LDU (owner / neighbour face) matrices: host construction, summation order
// and the synthetic hexahedral mesh.
//
// The reference's LDUMatrix (matrix/details/ldu/LDUMatrix.cpp:42-168) sums a
// row as diag * x, then its owned faces in face order (upper coefficients,
// x at upperAddr), then the faces it neighbours in losort order (lower
// coefficients, x at lowerAddr). Here an LDU matrix is stored like a CRS
// matrix (same tile layout, tile-local CRS, level sets), and each entry
// carries its rank in that summation order, so the device SpMV and residual
// kernels, which sum a row's stored slots in order, reproduce the LDU sums
// bit for bit.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "host_matrix.hpp"

namespace gr {

std::shared_ptr<HostMatrix> HostMatrix::fromLdu(i64 n, i64 numFaces, const i64* owner, const i64* neighbour,
                                                const double* diag, const double* lower, const double* upper,
                                                i64 numTiles, gr_partitioner part, const i32* rowToTileIn,
                                                const double* coords, DType valueType) {
  if (n <= 0) fail(GR_EINVAL, "matrix must have at least one cell");
  if (numFaces < 0) fail(GR_EINVAL, "num_faces must not be negative");
  if (!diag || (numFaces > 0 && (!owner || !neighbour || !lower)))
    fail(GR_EINVAL, "owner, neighbour, lower and diag must not be NULL");
  // OpenFOAM's upper-triangular face order (LDUAddressing.hpp:42-91):
  // lowerAddr < upperAddr, faces grouped by owner (ownerStartAddr).
  for (i64 f = 0; f < numFaces; ++f) {
    if (owner[f] < 0 || neighbour[f] >= n || owner[f] >= neighbour[f])
      fail(GR_EINVAL, "face " + std::to_string(f) + ": need 0 <= owner < neighbour < num_cells");
    if (f > 0 && owner[f] < owner[f - 1])
      fail(GR_EINVAL, "faces must be sorted by owner (face " + std::to_string(f) + ")");
  }
  Coo coo;
  coo.nrows = coo.ncols = n;
  coo.row.reserve(n + 2 * numFaces);
  coo.col.reserve(n + 2 * numFaces);
  coo.val.reserve(n + 2 * numFaces);
  for (i64 c = 0; c < n; ++c) {
    coo.row.push_back(c);
    coo.col.push_back(c);
    coo.val.push_back(diag[c]);
  }
  for (i64 f = 0; f < numFaces; ++f) {
    coo.row.push_back(owner[f]);
    coo.col.push_back(neighbour[f]);
    coo.val.push_back(upper ? upper[f] : lower[f]);
    coo.row.push_back(neighbour[f]);
    coo.col.push_back(owner[f]);
    coo.val.push_back(lower[f]);
  }
  // fromCoo rejects duplicate faces (a repeated (owner, neighbour) pair).
  auto A = fromCoo(std::move(coo), numTiles, part, rowToTileIn, coords, valueType);
  auto round = [&](double v) { return valueType == DType::F32 ? static_cast<double>(static_cast<float>(v)) : v; };
  A->format = GR_FORMAT_LDU;
  A->lduOwner.assign(owner, owner + numFaces);
  A->lduNeighbour.assign(neighbour, neighbour + numFaces);
  A->lduLower.resize(numFaces);
  A->lduUpper.resize(numFaces);
  A->lduDiag.resize(n);
  for (i64 f = 0; f < numFaces; ++f) {
    A->lduLower[f] = round(lower[f]);
    A->lduUpper[f] = round(upper ? upper[f] : lower[f]);
  }
  for (i64 c = 0; c < n; ++c) A->lduDiag[c] = round(diag[c]);

  // Per cell: owned faces are [ownerStart[c], ownerStart[c+1]); the faces it
  // neighbours, in losort order (by neighbour, then face index), are
  // losort[losortStart[c] .. losortStart[c+1]).
  std::vector<i64> ownerStart(n + 1, 0), losortStart(n + 1, 0), losort(numFaces);
  for (i64 f = 0; f < numFaces; ++f) {
    ownerStart[owner[f] + 1]++;
    losortStart[neighbour[f] + 1]++;
  }
  for (i64 c = 0; c < n; ++c) {
    ownerStart[c + 1] += ownerStart[c];
    losortStart[c + 1] += losortStart[c];
  }
  {
    std::vector<i64> fill(losortStart.begin(), losortStart.end() - 1);
    for (i64 f = 0; f < numFaces; ++f) losort[fill[neighbour[f]]++] = f;
  }
  HostMatrix& H = *A;
  H.sumRank.assign(H.m, 0);
  parallelChunks(n, [&](i64 b, i64 e) {
    std::vector<i64> seq;
    for (i64 r = b; r < e; ++r) {
      const i64 c = H.iperm[r];
      seq.clear();
      for (i64 f = ownerStart[c]; f < ownerStart[c + 1]; ++f) seq.push_back(neighbour[f]);
      for (i64 s = losortStart[c]; s < losortStart[c + 1]; ++s) seq.push_back(owner[losort[s]]);
      if (static_cast<i64>(seq.size()) != H.rowPtr[r + 1] - H.rowPtr[r])
        fail(GR_EINVAL, "LDU faces and stored entries disagree for cell " + std::to_string(c));
      for (i64 p = H.rowPtr[r]; p < H.rowPtr[r + 1]; ++p) {
        const i64 gc = H.iperm[H.colPerm[p]];
        const auto it = std::find(seq.begin(), seq.end(), gc);
        H.sumRank[p] = static_cast<i32>(it - seq.begin());
      }
    }
  });
  return A;
}

LduMesh generateLduMesh(i64 nx, i64 ny, i64 nz, uint64_t jitterSeed, uint64_t permSeed, uint64_t coefSeed) {
  if (nx <= 0 || ny <= 0 || nz <= 0) fail(GR_EINVAL, "grid dimensions must be positive");
  LduMesh M;
  const i64 n = nx * ny * nz;
  M.n = n;
  // Cell ids: a Fisher-Yates shuffle driven by the counter-based stream.
  std::vector<i64> id(n);
  std::iota(id.begin(), id.end(), i64(0));
  {
    std::vector<double> u(std::max<i64>(n - 1, 1));
    generateUniform(permSeed, n - 1, 0.0, 1.0, u.data());
    for (i64 i = n - 1; i > 0; --i) {
      i64 j = static_cast<i64>(u[n - 1 - i] * static_cast<double>(i + 1));
      if (j > i) j = i;
      std::swap(id[i], id[j]);
    }
  }
  // Faces between neighbouring cells, owner = smaller id.
  std::vector<std::pair<i64, i64>> faces;
  faces.reserve(3 * n);
  for (i64 k = 0; k < nz; ++k)
    for (i64 j = 0; j < ny; ++j)
      for (i64 i = 0; i < nx; ++i) {
        const i64 g = i + nx * (j + ny * k);
        auto add = [&](i64 g2) {
          const i64 a = id[g], b = id[g2];
          faces.emplace_back(std::min(a, b), std::max(a, b));
        };
        if (i + 1 < nx) add(g + 1);
        if (j + 1 < ny) add(g + nx);
        if (k + 1 < nz) add(g + nx * ny);
      }
  std::sort(faces.begin(), faces.end());
  const i64 F = static_cast<i64>(faces.size());
  M.owner.resize(F);
  M.neighbour.resize(F);
  std::vector<double> u(F);
  generateUniform(coefSeed, F, -2.0, 2.0, u.data());
  M.lower.resize(F);
  M.diag.assign(n, 1e-3);
  std::vector<double> sum(n, 0.0);
  for (i64 f = 0; f < F; ++f) {
    M.owner[f] = faces[f].first;
    M.neighbour[f] = faces[f].second;
    const double c = std::pow(10.0, u[f]);
    M.lower[f] = -c;
    sum[faces[f].first] += c;
    sum[faces[f].second] += c;
  }
  for (i64 c = 0; c < n; ++c) M.diag[c] = sum[c] + 1e-3;
  M.upper = M.lower;
  // Cell centroids of the jittered node positions.
  const i64 mx = nx + 1, my = ny + 1, mz = nz + 1;
  std::vector<double> jit(3 * mx * my * mz);
  generateUniform(jitterSeed, static_cast<i64>(jit.size()), -0.2, 0.2, jit.data());
  M.coords.assign(3 * n, 0.0);
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 g = b; g < e; ++g) {
      const i64 i = g % nx, j = (g / nx) % ny, k = g / (nx * ny);
      double acc[3] = {0, 0, 0};
      for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
          for (int dx = 0; dx < 2; ++dx) {
            const i64 node = (i + dx) + mx * ((j + dy) + my * (k + dz));
            acc[0] += static_cast<double>(i + dx) + jit[3 * node];
            acc[1] += static_cast<double>(j + dy) + jit[3 * node + 1];
            acc[2] += static_cast<double>(k + dz) + jit[3 * node + 2];
          }
      for (int d = 0; d < 3; ++d) M.coords[3 * id[g] + d] = acc[d] / 8.0;
    }
  });
  return M;
}

}  // namespace gr
